// complex16 (k-point) hpsi: u_k storage, k entering through zcoef_kin and const_k2.
//
// Reference: z_op_kinetic_sol flag_nab branch (src/kinetic/d_kinetic_sol_module.f90:144-200;
// the z_ module is the same text on complex arrays):
//   H u(i) = (coef_lap0 + const_k2 + Vloc) u(i)
//          + sum_d sum_m [ zcoef_kin(d,m) u(i + m e_d) + conj(zcoef_kin(d,m)) u(i - m e_d) ],
//   zcoef_kin(d,+m) = coef_lap(d,m) - i coef_nabk(d,m)  (src/kinetic/kinetic_module.f90:155-159),
// periodic wrap of u (no Bloch phase in the halo), and the nonlocal part
// z_op_ps_nloc_mr (src/ps_nloc_mr_module.f90:1260-1359): gather with conj(z_uVk), scatter
// with z_uVk.  The stencil is the warp-specialised streaming kernel of hpsi_ws.cu in its
// complex form (a grid point is an interleaved (re, im) pair); this file holds the gather
// (+ Dij) before it and the scatter after it.
#include "stencil.cuh"

namespace rsdft {

// gather with conj(uVk) (pre-conjugated weights) + Dij: coef[b][lma] (interleaved complex)
template <typename S, int PG, int BB>
__global__ void __launch_bounds__(256) k_nl_gather_cplx(const S* __restrict__ psi, long long ld, int nb,
                                                        const int* __restrict__ gofs, const int* __restrict__ gjj,
                                                        const S* __restrict__ gw, const int* __restrict__ gplist,
                                                        const double* __restrict__ gD, double dV, S* coef, int ldc) {
  const int g = blockIdx.x;
  const int b0 = blockIdx.y * BB;
  const int f0 = gofs[g], f1 = gofs[g + 1];
  S accr[BB][PG], acci[BB][PG];
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) accr[bb][p] = acci[bb][p] = S(0);
  for (int j = f0 + threadIdx.x; j < f1; j += blockDim.x) {
    const int idx = __ldg(gjj + j);
    S wr[PG], wi[PG];
#pragma unroll
    for (int p = 0; p < PG; ++p) {
      wr[p] = __ldg(gw + ((size_t)j * PG + p) * 2);
      wi[p] = __ldg(gw + ((size_t)j * PG + p) * 2 + 1);
    }
#pragma unroll
    for (int bb = 0; bb < BB; ++bb) {
      if (b0 + bb < nb) {
        const S xr = __ldg(psi + (long long)(b0 + bb) * ld + 2 * (long long)idx);
        const S xi = __ldg(psi + (long long)(b0 + bb) * ld + 2 * (long long)idx + 1);
#pragma unroll
        for (int p = 0; p < PG; ++p) {
          accr[bb][p] += wr[p] * xr - wi[p] * xi;
          acci[bb][p] += wr[p] * xi + wi[p] * xr;
        }
      }
    }
  }
  __shared__ S red[8][2 * BB * PG];
  __shared__ double u[2 * BB * PG];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) {
      S x = accr[bb][p], y = acci[bb][p];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_xor_sync(0xffffffffu, x, o);
        y += __shfl_xor_sync(0xffffffffu, y, o);
      }
      if (lane == 0) {
        red[wid][2 * (bb * PG + p)] = x;
        red[wid][2 * (bb * PG + p) + 1] = y;
      }
    }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (threadIdx.x < 2 * BB * PG) {
    double t = 0.0;
    for (int w2 = 0; w2 < nw; ++w2) t += (double)red[w2][threadIdx.x];
    u[threadIdx.x] = t * dV;
  }
  __syncthreads();
  if (threadIdx.x < BB * PG) {
    const int bb = threadIdx.x / PG, p = threadIdx.x % PG;
    (void)gplist;
    if (b0 + bb < nb) {
      double cr = 0.0, ci = 0.0;
#pragma unroll
      for (int q = 0; q < PG; ++q) {
        const double d = gD[((size_t)g * PG + p) * PG + q];
        cr += d * u[2 * (bb * PG + q)];
        ci += d * u[2 * (bb * PG + q) + 1];
      }
      coef[((long long)(b0 + bb) * ldc + g * PG + p) * 2] = (S)cr;
      coef[((long long)(b0 + bb) * ldc + g * PG + p) * 2 + 1] = (S)ci;
    }
  }
}

template <typename S, int PG, int BB>
static void launch_gather_c(Ctx& c, const S* psi, size_t ld, int nb, S* coef, const S* gw) {
  NonlocalTables& nl = c.nl;
  dim3 grid(nl.ngroups, (nb + BB - 1) / BB);
  k_nl_gather_cplx<S, PG, BB><<<grid, 256, 0, c.stream>>>(psi, (long long)ld, nb, nl.gofs.as<int>(), nl.gjj.as<int>(),
                                                           gw, nl.gplist.as<int>(), nl.gD.as<double>(), c.p.dv, coef,
                                                           nl.ngroups * PG);
  c.launches++;
}

// Nonlocal scatter of the complex build after the stencil: out_b[pt] += sum over the point's
// records r of uVk_r . c_b[atom_r] (complex; src/ps_nloc_mr_module.f90:1341, the z_uVk scatter).
// One thread per covered grid point, bands looped inside the CTA four at a time.
template <typename S>
__global__ void __launch_bounds__(256) k_nl_scatter_c(const int* __restrict__ cov, int ncov,
                                                      const int* __restrict__ rowptr, const int* __restrict__ rg,
                                                      const S* __restrict__ ru, int pg, const S* __restrict__ coef,
                                                      int ldc, S* __restrict__ out, long long ld, int nb, int bchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncov) return;
  const int pt = __ldg(cov + i);
  const int r0 = __ldg(rowptr + pt), r1 = __ldg(rowptr + pt + 1);
  const int b0 = blockIdx.y * bchunk, b1 = min(nb, b0 + bchunk);
  constexpr int BU = 4;
  for (int b = b0; b < b1; b += BU) {
    S ar[BU], ai[BU];
#pragma unroll
    for (int u = 0; u < BU; ++u) ar[u] = ai[u] = S(0);
    for (int r = r0; r < r1; ++r) {
      const S* uv = ru + 2 * (size_t)r * pg;
      const size_t go = 2 * (size_t)__ldg(rg + r) * pg;
      for (int q = 0; q < pg; ++q) {
        const S ur = __ldg(uv + 2 * q), ui = __ldg(uv + 2 * q + 1);
#pragma unroll
        for (int u = 0; u < BU; ++u) {
          if (b + u >= b1) break;
          const S* cc = coef + 2 * (size_t)(b + u) * ldc + go + 2 * q;
          const S cr = __ldg(cc), ci = __ldg(cc + 1);
          ar[u] = ::fma(ur, cr, ::fma(-ui, ci, ar[u]));
          ai[u] = ::fma(ur, ci, ::fma(ui, cr, ai[u]));
        }
      }
    }
#pragma unroll
    for (int u = 0; u < BU; ++u)
      if (b + u < b1) {
        S* o = out + (size_t)(b + u) * ld + 2 * (size_t)pt;
        o[0] += ar[u];
        o[1] += ai[u];
      }
  }
}

template <typename S>
static int nl_scatter_c(Ctx& c, int k, const S* coef, S* out, size_t ld, int nb) {
  const NonlocalTables& nl = c.nl;
  if (nl.ncov == 0 || nb <= 0) return 0;
  const S* ru = std::is_same<S, double>::value ? (const S*)nl.perk[k].ru64.as<double>()
                                               : (const S*)nl.perk[k].ru32.as<float>();
  const int ldc = nl.ngroups * nl.pg;
  const int bchunk = 16;
  const dim3 grid((nl.ncov + 255) / 256, (nb + bchunk - 1) / bchunk);
  ProfScope ps(c, "nl_scatter",
               (double)nb * nl.ncov * 4.0 * sizeof(S) + (double)nl.nrec * (4 + 2 * nl.pg * sizeof(S)));
  k_nl_scatter_c<S><<<grid, 256, 0, c.stream>>>(nl.cov.as<int>(), nl.ncov, nl.rec_rowptr.as<int>(), nl.rec_g.as<int>(),
                                                ru, nl.pg, coef, ldc, out, (long long)ld, nb, bchunk);
  c.launches++;
  return check_launch("nl_scatter_cplx");
}

// psi/hpsi interleaved complex; ld in S units (2 x complex leading dimension)
template <typename S>
int hpsi_cplx(Ctx& c, int k, int s, const S* psi, S* out, size_t ld, int nb) {
  RS_CHECK(c.cplx, RSDFT_ERR_STATE, "complex hpsi called on a real8 context");
  RS_CHECK(c.kp[k].set, RSDFT_ERR_STATE, "k-point %d not set", k + 1);
  RS_CHECK(c.vloc_set[s], RSDFT_ERR_STATE, "Vloc for spin %d not set", s + 1);
  if (nb <= 0) return 0;
  S* coef = nullptr;
  if (c.nl.nproj > 0) {
    RS_TRY(nl_prepare_k(c, k));
    RS_TRY(c.ws_coef.ensure((size_t)nb * c.nl.ngroups * c.nl.pg * 2 * sizeof(S)));
    coef = c.ws_coef.as<S>();
    const S* gw = std::is_same<S, double>::value ? (const S*)c.nl.perk[k].gw64.as<double>()
                                                 : (const S*)c.nl.perk[k].gw32.as<float>();
    ProfScope ps(c, "nl_gather");
    switch (c.nl.pg) {
      case 1: launch_gather_c<S, 1, 8>(c, psi, ld, nb, coef, gw); break;
      case 4: launch_gather_c<S, 4, 4>(c, psi, ld, nb, coef, gw); break;
      case 9: launch_gather_c<S, 9, 2>(c, psi, ld, nb, coef, gw); break;
      case 16: launch_gather_c<S, 16, 1>(c, psi, ld, nb, coef, gw); break;
      default: RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "projectors per atom > 16 not built in");
    }
    RS_TRY(check_launch("nl_gather_cplx"));
  }
  if (c.p.md == 6)
    RS_TRY((launch_stencil_ws_c<S, 6>(c, k, s, psi, out, ld, nb)));
  else if (c.p.md == 4)
    RS_TRY((launch_stencil_ws_c<S, 4>(c, k, s, psi, out, ld, nb)));
  else
    RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
  return coef ? nl_scatter_c<S>(c, k, coef, out, ld, nb) : 0;
}
template int hpsi_cplx<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_cplx<double>(Ctx&, int, int, const double*, double*, size_t, int);

}  // namespace rsdft
