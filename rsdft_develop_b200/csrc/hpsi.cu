// Many-band hpsi for the real8 (Gamma) build: H psi = T psi + Vloc psi + V_NL psi.
//
// Reference semantics (restated, not translated):
//   kinetic + Vloc  src/kinetic/d_kinetic_sol_module.f90:244-292  (Md=6 star stencil,
//                   (coef_lap0 + Vloc) on the centre, periodic halo src/bc/bcset_3_module.f90)
//   nonlocal        src/ps_nloc_mr_module.f90:1159-1258 (gather uVunk = dV sum uVk psi(JJP),
//                   Dij pairs, scatter psi(JJP) += uVk * sum Dij uVunk); the KB form
//                   src/d_ps_nloc2_op_module.f90:146-288 is the diagonal-Dij case.
//
// This file holds the host side of hpsi, the atom-centred gather and the nonlocal scatter: the
// projector gather + Dij runs first and writes the coefficient rows c_b (atom-major,
// PG-padded); the stencil with V_loc is the persistent streaming kernel of hpsi_stream.cu;
// the scatter then adds uV . c_b at every covered grid point (or, selectable, the stencil adds
// it from records staged per plane).
#include "stencil.cuh"

namespace rsdft {

// ---------------------------------------------------------------------------
// nonlocal gather + Dij (atom-centred):
//   c_b[g*PG + p] = sum_q D_g[p][q] dV sum_j uV_g(j,q) psi_b(JJ_g(j))
// ---------------------------------------------------------------------------
template <typename T, int PG, int BB>
__global__ void __launch_bounds__(256) k_nl_gather_real(const T* __restrict__ psi, long long ld, int nb,
                                                        const int* __restrict__ gofs, const int* __restrict__ gjj,
                                                        const T* __restrict__ gw, const double* __restrict__ gD,
                                                        double dV, T* coef, int ldc) {
  const int g = blockIdx.x;
  const int b0 = blockIdx.y * BB;
  const int f0 = gofs[g], f1 = gofs[g + 1];
  T acc[BB][PG];
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) acc[bb][p] = T(0);
  for (int j = f0 + threadIdx.x; j < f1; j += blockDim.x) {
    const int idx = __ldg(gjj + j);
    T w[PG];
#pragma unroll
    for (int p = 0; p < PG; ++p) w[p] = __ldg(gw + (size_t)j * PG + p);
#pragma unroll
    for (int bb = 0; bb < BB; ++bb) {
      if (b0 + bb < nb) {
        const T v = __ldg(psi + (long long)(b0 + bb) * ld + idx);
#pragma unroll
        for (int p = 0; p < PG; ++p) acc[bb][p] += w[p] * v;
      }
    }
  }
  __shared__ T red[8][BB * PG];
  __shared__ double u[BB * PG];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) {
      T x = acc[bb][p];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) red[wid][bb * PG + p] = x;
    }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (threadIdx.x < BB * PG) {
    double t = 0.0;
    for (int w2 = 0; w2 < nw; ++w2) t += (double)red[w2][threadIdx.x];
    u[threadIdx.x] = t * dV;
  }
  __syncthreads();
  if (threadIdx.x < BB * PG) {
    const int bb = threadIdx.x / PG, p = threadIdx.x % PG;
    if (b0 + bb < nb) {
      double cfs = 0.0;
#pragma unroll
      for (int q = 0; q < PG; ++q) cfs += gD[((size_t)g * PG + p) * PG + q] * u[bb * PG + q];
      coef[(long long)(b0 + bb) * ldc + g * PG + p] = (T)cfs;
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <typename T, int PG, int BB>
static void launch_gather(Ctx& c, const T* psi, size_t ld, int nb, T* coef, const T* gw) {
  NonlocalTables& nl = c.nl;
  dim3 grid(nl.ngroups, (nb + BB - 1) / BB);
  k_nl_gather_real<T, PG, BB><<<grid, 256, 0, c.stream>>>(psi, (long long)ld, nb, nl.gofs.as<int>(), nl.gjj.as<int>(),
                                                           gw, nl.gD.as<double>(), c.p.dv, coef, nl.ngroups * PG);
  c.launches++;
}

template <typename T>
static int nl_gather(Ctx& c, int k, const T* psi, size_t ld, int nb, T* coef) {
  NonlocalTables& nl = c.nl;
  const T* gw = std::is_same<T, double>::value ? nl.perk[k].gw64.as<T>() : nl.perk[k].gw32.as<T>();
  const double bytes = (double)sizeof(T) * nl.ftotal * ((double)nb + nl.pg) + 4.0 * nl.ftotal;
  ProfScope ps(c, "nl_gather", bytes);
  switch (nl.pg) {
    case 1: launch_gather<T, 1, 8>(c, psi, ld, nb, coef, gw); break;
    case 4: launch_gather<T, 4, 8>(c, psi, ld, nb, coef, gw); break;
    case 9: launch_gather<T, 9, 4>(c, psi, ld, nb, coef, gw); break;
    case 16: launch_gather<T, 16, 2>(c, psi, ld, nb, coef, gw); break;
    default: RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "projectors per atom > 16 not built in");
  }
  return check_launch("nl_gather");
}

int record_segment_max(Ctx& c, int tile_y) {
  auto it = c.nl.seg_max.find(tile_y);
  if (it != c.nl.seg_max.end()) return it->second;
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  int mx = 0;
  const std::vector<int>& rp = c.nl.h_rowptr;
  for (int p = 0; p < n3; ++p)
    for (int y0 = 0; y0 < n2; y0 += tile_y) {
      const size_t b0 = ((size_t)p * n2 + y0) * n1, b1 = b0 + (size_t)std::min(tile_y, n2 - y0) * n1;
      mx = std::max(mx, rp[b1] - rp[b0]);
    }
  c.nl.seg_max.emplace(tile_y, mx);
  return mx;
}

// ---------------------------------------------------------------------------
// nonlocal scatter after the stencil: out_b[pt] += sum over the point's records r
// uV_r . c_b[atom_r] (src/ps_nloc_mr_module.f90:1159-1258, the psi(JJP) += uVk ... update).
// One thread per grid point that some projector reaches (the covered list, ascending), bands
// looped inside the CTA so the point's few records stay in L1; one read-modify-write of H psi
// per covered point and band.
// ---------------------------------------------------------------------------
template <typename T, int PG>
__global__ void __launch_bounds__(256) k_nl_scatter(const int* __restrict__ cov, int ncov,
                                                    const int* __restrict__ rowptr, const int* __restrict__ rg,
                                                    const T* __restrict__ ru, int pgr, const T* __restrict__ coef,
                                                    int ldc, T* __restrict__ out, long long ld, int nb, int bchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncov) return;
  const int pt = __ldg(cov + i);
  const int r0 = __ldg(rowptr + pt), r1 = __ldg(rowptr + pt + 1);
  const int b0 = blockIdx.y * bchunk, b1 = min(nb, b0 + bchunk);
  const int np = PG > 0 ? PG : pgr;
  constexpr int BU = 4;  // bands in flight per thread (8 measured no faster)
  for (int b = b0; b < b1; b += BU) {
    T acc[BU], cur[BU];
#pragma unroll
    for (int u = 0; u < BU; ++u) {
      acc[u] = T(0);
      cur[u] = b + u < b1 ? out[(size_t)(b + u) * ld + pt] : T(0);
    }
    for (int r = r0; r < r1; ++r) {
      const T* uv = ru + (size_t)r * np;
      const size_t go = (size_t)__ldg(rg + r) * np;
#pragma unroll
      for (int u = 0; u < BU; ++u) {
        if (b + u >= b1) break;
        const T* cc = coef + (size_t)(b + u) * ldc + go;
#pragma unroll
        for (int q = 0; q < (PG > 0 ? PG : 1); ++q) acc[u] = ::fma(__ldg(uv + q), __ldg(cc + q), acc[u]);
        if (PG == 0)
          for (int q = 1; q < np; ++q) acc[u] = ::fma(__ldg(uv + q), __ldg(cc + q), acc[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < BU; ++u)
      if (b + u < b1) out[(size_t)(b + u) * ld + pt] = cur[u] + acc[u];
  }
}

template <typename T>
static int nl_scatter(Ctx& c, int k, const T* coef, T* out, size_t ld, int nb) {
  const NonlocalTables& nl = c.nl;
  if (nl.ncov == 0 || nb <= 0) return 0;
  const T* ru = std::is_same<T, double>::value ? (const T*)nl.perk[k].ru64.as<double>()
                                               : (const T*)nl.perk[k].ru32.as<float>();
  const int ldc = nl.ngroups * nl.pg;
  const int bchunk = 16;
  const dim3 grid((nl.ncov + 255) / 256, (nb + bchunk - 1) / bchunk);
  ProfScope ps(c, "nl_scatter", (double)nb * nl.ncov * 2.0 * sizeof(T) + (double)nl.nrec * (4 + nl.pg * sizeof(T)));
  if (nl.pg == 4)
    k_nl_scatter<T, 4><<<grid, 256, 0, c.stream>>>(nl.cov.as<int>(), nl.ncov, nl.rec_rowptr.as<int>(),
                                                    nl.rec_g.as<int>(), ru, nl.pg, coef, ldc, out, (long long)ld, nb,
                                                    bchunk);
  else
    k_nl_scatter<T, 0><<<grid, 256, 0, c.stream>>>(nl.cov.as<int>(), nl.ncov, nl.rec_rowptr.as<int>(),
                                                    nl.rec_g.as<int>(), ru, nl.pg, coef, ldc, out, (long long)ld, nb,
                                                    bchunk);
  c.launches++;
  return check_launch("nl_scatter");
}

// vloc_override / c0_shift: the kinetic-only operator (T + shift) used for training targets.
// With coef the nonlocal term is added: by the separate scatter kernel after the stencil
// (default), or inside the stencil (c.nl_fused).
template <typename T, int MD>
static int launch_stencil(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef,
                          const T* vloc_override = nullptr, double c0_shift = 0.0, bool allow_fused = true) {
  if (coef != nullptr && c.nl_fused && allow_fused)
    return launch_stencil_stream<T, MD>(c, k, s, psi, out, ld, nb, coef, vloc_override, c0_shift);
  RS_TRY((launch_stencil_ws<T, MD>(c, k, s, psi, out, ld, nb, vloc_override, c0_shift)));
  return coef ? nl_scatter<T>(c, k, coef, out, ld, nb) : 0;
}

template <typename T>
int hpsi_real(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "real hpsi called on a complex16 context");
  RS_CHECK(c.kp[k].set || c.p.nk == 1, RSDFT_ERR_STATE, "k-point %d not set", k + 1);
  RS_CHECK(c.vloc_set[s], RSDFT_ERR_STATE, "Vloc for spin %d not set", s + 1);
  if (nb <= 0) return 0;
  T* coef = nullptr;
  if (c.nl.nproj > 0) {
    RS_TRY(nl_prepare_k(c, k));
    RS_TRY(c.ws_coef.ensure((size_t)nb * c.nl.ngroups * c.nl.pg * sizeof(T)));
    coef = c.ws_coef.as<T>();
    RS_TRY(nl_gather<T>(c, k, psi, ld, nb, coef));
  }
  if (c.p.md == 6) return launch_stencil<T, 6>(c, k, s, psi, out, ld, nb, coef);
  if (c.p.md == 4) return launch_stencil<T, 4>(c, k, s, psi, out, ld, nb, coef);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}

template int hpsi_real<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_real<double>(Ctx&, int, int, const double*, double*, size_t, int);

// hpsi with caller-provided scratch for the nonlocal coefficient rows (coef_cap elements of
// T); performs no device allocation.  Always the stencil + scatter form: it needs no tuning
// runs and no host synchronisation.
template <typename T>
int hpsi_real_scratch(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, T* coef, size_t coef_cap) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "real hpsi called on a complex16 context");
  RS_CHECK(c.kp[k].set || c.p.nk == 1, RSDFT_ERR_STATE, "k-point %d not set", k + 1);
  RS_CHECK(c.vloc_set[s], RSDFT_ERR_STATE, "Vloc for spin %d not set", s + 1);
  if (nb <= 0) return 0;
  T* cf = nullptr;
  if (c.nl.nproj > 0) {
    RS_TRY(nl_prepare_k(c, k));
    const size_t need = (size_t)nb * c.nl.ngroups * c.nl.pg;
    RS_CHECK(coef != nullptr && need <= coef_cap, RSDFT_ERR_ARG,
             "nonlocal scratch too small: %zu coefficients needed, %zu available", need, coef_cap);
    cf = coef;
    RS_TRY(nl_gather<T>(c, k, psi, ld, nb, cf));
  }
  if (c.p.md == 6) return launch_stencil<T, 6>(c, k, s, psi, out, ld, nb, cf, nullptr, 0.0, false);
  if (c.p.md == 4) return launch_stencil<T, 4>(c, k, s, psi, out, ld, nb, cf, nullptr, 0.0, false);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}
template int hpsi_real_scratch<double>(Ctx&, int, int, const double*, double*, size_t, int, double*, size_t);

// y = (T + shift) x with T the finite-difference kinetic operator alone (no V_loc, no
// projectors), real Gamma build, FP32.
int kinetic_shifted(Ctx& c, const float* x, float* y, size_t ld, int nb, double shift) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "kinetic_shifted: real build only");
  if (nb <= 0) return 0;
  if (!c.vzero.p || c.vzero.bytes < sizeof(float) * c.ng) {
    RS_TRY(c.vzero.ensure(sizeof(float) * c.ng));
    RS_CUDA(cudaMemsetAsync(c.vzero.p, 0, sizeof(float) * c.ng, c.stream));
  }
  const float* vz = c.vzero.as<float>();
  if (c.p.md == 6) return launch_stencil<float, 6>(c, 0, 0, x, y, ld, nb, nullptr, vz, shift);
  if (c.p.md == 4) return launch_stencil<float, 4>(c, 0, 0, x, y, ld, nb, nullptr, vz, shift);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}

}  // namespace rsdft
