// complex16 (k-point) hpsi: u_k storage, k entering through zcoef_kin and const_k2.
//
// Reference: z_op_kinetic_sol flag_nab branch (src/kinetic/d_kinetic_sol_module.f90:144-200;
// the z_ module is the same text on complex arrays):
//   H u(i) = (coef_lap0 + const_k2 + Vloc) u(i)
//          + sum_d sum_m [ zcoef_kin(d,m) u(i + m e_d) + conj(zcoef_kin(d,m)) u(i - m e_d) ],
//   zcoef_kin(d,+m) = coef_lap(d,m) - i coef_nabk(d,m)  (src/kinetic/kinetic_module.f90:155-159),
// periodic wrap of u (no Bloch phase in the halo), and the nonlocal part
// z_op_ps_nloc_mr (src/ps_nloc_mr_module.f90:1260-1359): gather with conj(z_uVk), scatter
// with z_uVk.  Same streaming design as the real kernel in hpsi.cu; a grid point is an
// interleaved (re, im) pair.
#include "ctx.cuh"
#include "ptx.cuh"

namespace rsdft {

template <typename S> struct CVec;
template <> struct CVec<float> { static constexpr int V = 2; using type = float4; };
template <> struct CVec<double> { static constexpr int V = 1; using type = double2; };

// load/store V complex points (16 bytes)
template <typename S, int V>
__device__ __forceinline__ void cld(const S* p, S (&re)[V], S (&im)[V]) {
  using VT = typename CVec<S>::type;
  VT t = *reinterpret_cast<const VT*>(p);
  const S* tt = reinterpret_cast<const S*>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) {
    re[i] = tt[2 * i];
    im[i] = tt[2 * i + 1];
  }
}
template <typename S, int V>
__device__ __forceinline__ void cst(S* p, const S (&re)[V], const S (&im)[V]) {
  using VT = typename CVec<S>::type;
  VT t;
  S* tt = reinterpret_cast<S*>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) {
    tt[2 * i] = re[i];
    tt[2 * i + 1] = im[i];
  }
  *reinterpret_cast<VT*>(p) = t;
}

__device__ __forceinline__ int pmodc(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

template <typename S, int MD>
struct StArgsC {
  const S* psi;   // interleaved, band stride ld (in S units)
  S* out;
  long long ld;
  const S* vloc;  // real, ng
  int n1, n2, n3;
  int tile_y, tz, stage_elems;  // stage_elems in S units
  S c0;
  S cc[3][MD], cs[3][MD];       // zcoef_kin(d,+m) = cc - i cs
  const int* rowptr;  // per point: scatter records [rowptr[i], rowptr[i+1])
  const int* rec_g;   // record -> atom group
  const S* val;       // record -> interleaved uVk of the group's projectors [pg]
  int pg;
  const S* coef;   // interleaved c[b][p]
  int ldc;         // complex elements per band in coef
  unsigned* status;
};

constexpr uint32_t kWaitPollsC = 1u << 22;

template <typename S, int MD, int R, int SS>
__global__ void __launch_bounds__(256) k_stencil_cplx(const StArgsC<S, MD> a) {
  constexpr int V = CVec<S>::V;
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + V - 1) / V;
  extern __shared__ __align__(128) unsigned char smem[];
  S* stages = reinterpret_cast<S*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + (size_t)SS * a.stage_elems * sizeof(S));
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const int x0 = threadIdx.x * V;
  const int yl = threadIdx.y * R;
  const int y0 = blockIdx.x * a.tile_y;
  const int z0 = blockIdx.y * a.tz;
  const int zend = min(z0 + a.tz, n3);
  const int rows = a.tile_y + 2 * MD;
  const int nplanes = (zend - z0) + 2 * MD;
  const S* src = a.psi + (long long)blockIdx.z * a.ld;
  S* dst = a.out + (long long)blockIdx.z * a.ld;
  const S* coefb = a.coef ? a.coef + (long long)blockIdx.z * 2 * a.ldc : nullptr;
  const int rowS = 2 * n1;  // S units per staged row

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < SS; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int q) {
    const int zg = pmodc(z0 - MD + q, n3);
    S* st = stages + (size_t)(q % SS) * a.stage_elems;
    uint64_t* br = &bar[q % SS];
    mbar_arrive_expect_tx(br, (uint32_t)((size_t)rows * rowS * sizeof(S)));
    int r = 0;
    while (r < rows) {
      const int gy = pmodc(y0 - MD + r, n2);
      const int len = min(rows - r, n2 - gy);
      bulk_g2s(st + (size_t)r * rowS, src + ((size_t)zg * n2 + gy) * rowS, (uint32_t)((size_t)len * rowS * sizeof(S)),
               br);
      r += len;
    }
  };
  if (tid == 0)
    for (int q = 0; q < SS - 1 && q < nplanes; ++q) issue(q);

  bool rowok[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rowok[r] = (y0 + yl + r) < n2;
  S ar[NQ][R][V], ai[NQ][R][V];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < V; ++i) ar[q][r][i] = ai[q][r][i] = S(0);

  int issued_upto = min(SS - 1, nplanes);
  bool aborted = false;
  for (int qb = 0; qb < nplanes && !aborted; qb += NQ) {
#pragma unroll
    for (int s = 0; s < NQ; ++s) {
      const int q = qb + s;
      if (q < nplanes && !aborted) {
        if (tid == 0 && q + SS - 1 < nplanes) {
          fence_proxy_async_smem();
          issue(q + SS - 1);
          issued_upto = q + SS;
        }
        bool ok = mbar_wait_bounded(&bar[q % SS], (uint32_t)((q / SS) & 1), kWaitPollsC);
        if (__syncthreads_or(!ok)) {
          aborted = true;
          if (tid == 0) atomicOr(a.status, DEV_WAIT_TIMEOUT);
          break;
        }
        const S* pl = stages + (size_t)(q % SS) * a.stage_elems;
        const int p = z0 - MD + q;
        S vr[R][V], vi[R][V];
#pragma unroll
        for (int r = 0; r < R; ++r) cld<S, V>(pl + (size_t)(yl + r + MD) * rowS + 2 * x0, vr[r], vi[r]);
        if (p >= z0 && p < zend) {
          S tr[R][V], ti[R][V];
#pragma unroll
          for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int i = 0; i < V; ++i) {
              const S vl = rowok[r] ? __ldg(a.vloc + ((size_t)p * n2 + (y0 + yl + r)) * n1 + x0 + i) : S(0);
              tr[r][i] = (a.c0 + vl) * vr[r][i];
              ti[r][i] = (a.c0 + vl) * vi[r][i];
            }
            S wr[(2 * NCH + 1) * V], wi[(2 * NCH + 1) * V];
#pragma unroll
            for (int i = 0; i < V; ++i) {
              wr[NCH * V + i] = vr[r][i];
              wi[NCH * V + i] = vi[r][i];
            }
#pragma unroll
            for (int ch = 1; ch <= NCH; ++ch) {
              S lr[V], li[V], rr[V], ri[V];
              cld<S, V>(pl + (size_t)(yl + r + MD) * rowS + 2 * pmodc(x0 - ch * V, n1), lr, li);
              cld<S, V>(pl + (size_t)(yl + r + MD) * rowS + 2 * pmodc(x0 + ch * V, n1), rr, ri);
#pragma unroll
              for (int i = 0; i < V; ++i) {
                wr[(NCH - ch) * V + i] = lr[i];
                wi[(NCH - ch) * V + i] = li[i];
                wr[(NCH + ch) * V + i] = rr[i];
                wi[(NCH + ch) * V + i] = ri[i];
              }
            }
#pragma unroll
            for (int i = 0; i < V; ++i)
#pragma unroll
              for (int m = 1; m <= MD; ++m) {
                const S pr = wr[NCH * V + i + m], pi = wi[NCH * V + i + m];
                const S mr = wr[NCH * V + i - m], mi = wi[NCH * V + i - m];
                const S c = a.cc[0][m - 1], sn = a.cs[0][m - 1];
                tr[r][i] += c * (pr + mr) + sn * (pi - mi);
                ti[r][i] += c * (pi + mi) - sn * (pr - mr);
              }
          }
#pragma unroll
          for (int dy = -MD; dy < R + MD; ++dy) {
            S yr[V], yi[V];
            if (dy >= 0 && dy < R) {
#pragma unroll
              for (int i = 0; i < V; ++i) {
                yr[i] = vr[dy >= 0 && dy < R ? dy : 0][i];
                yi[i] = vi[dy >= 0 && dy < R ? dy : 0][i];
              }
            } else {
              cld<S, V>(pl + (size_t)(yl + dy + MD) * rowS + 2 * x0, yr, yi);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int m = dy - r;  // neighbour offset of row dy seen from output row r
              const int am = m > 0 ? m : -m;
              if (am >= 1 && am <= MD) {
                const S c = a.cc[1][(am >= 1 ? am : 1) - 1], sn = a.cs[1][(am >= 1 ? am : 1) - 1];
#pragma unroll
                for (int i = 0; i < V; ++i) {
                  if (m > 0) {  // zcoef * u
                    tr[r][i] += c * yr[i] + sn * yi[i];
                    ti[r][i] += c * yi[i] - sn * yr[i];
                  } else {      // conj(zcoef) * u
                    tr[r][i] += c * yr[i] - sn * yi[i];
                    ti[r][i] += c * yi[i] + sn * yr[i];
                  }
                }
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) {
              ar[s][r][i] += tr[r][i];
              ai[s][r][i] += ti[r][i];
            }
        }
        // z taps: plane p is the +m neighbour of output p-m and the -m neighbour of p+m
#pragma unroll
        for (int m = 1; m <= MD; ++m) {
          const S c = a.cc[2][m - 1], sn = a.cs[2][m - 1];
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) {
              ar[(s - m + NQ) % NQ][r][i] += c * vr[r][i] + sn * vi[r][i];
              ai[(s - m + NQ) % NQ][r][i] += c * vi[r][i] - sn * vr[r][i];
              ar[(s + m) % NQ][r][i] += c * vr[r][i] - sn * vi[r][i];
              ai[(s + m) % NQ][r][i] += c * vi[r][i] + sn * vr[r][i];
            }
        }
        {
          const int zo = p - MD;
          const int fs = (s + NQ - MD) % NQ;
          if (zo >= z0 && zo < zend) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
              if (rowok[r]) {
                S orr[V], oi[V];
#pragma unroll
                for (int i = 0; i < V; ++i) {
                  orr[i] = ar[fs][r][i];
                  oi[i] = ai[fs][r][i];
                }
                const size_t g = ((size_t)zo * n2 + (y0 + yl + r)) * n1 + x0;
                if (a.rowptr) {
                  const int e0 = __ldg(a.rowptr + g), eV = __ldg(a.rowptr + g + V);
                  if (e0 != eV) {
#pragma unroll
                    for (int i = 0; i < V; ++i) {
                      const int ea = __ldg(a.rowptr + g + i), eb = __ldg(a.rowptr + g + i + 1);
                      for (int e = ea; e < eb; ++e) {
                        // record e: atom group gg with its pg projector values uVk at this point
                        const int gg = __ldg(a.rec_g + e);
                        for (int q = 0; q < a.pg; ++q) {
                          const S ur = __ldg(a.val + 2 * ((size_t)e * a.pg + q));
                          const S ui = __ldg(a.val + 2 * ((size_t)e * a.pg + q) + 1);
                          const S cr = __ldg(coefb + 2 * (gg * a.pg + q)), ci = __ldg(coefb + 2 * (gg * a.pg + q) + 1);
                          orr[i] += ur * cr - ui * ci;
                          oi[i] += ur * ci + ui * cr;
                        }
                      }
                    }
                  }
                }
                cst<S, V>(dst + 2 * g, orr, oi);
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) ar[fs][r][i] = ai[fs][r][i] = S(0);
        }
        __syncthreads();
      }
    }
  }
  if (aborted && tid == 0)
    for (int q = 0; q < issued_upto; ++q) mbar_wait_bounded(&bar[q % SS], (uint32_t)((q / SS) & 1), kWaitPollsC);
}

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

template <typename S, int MD>
static int launch_stencil_c(Ctx& c, int k, int s, const S* psi, S* out, size_t ld, int nb, const S* coef) {
  constexpr int V = CVec<S>::V;
  constexpr int R = 2;
  constexpr int SS = 4;
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  RS_CHECK(n1 % V == 0 && n1 / V <= 256, RSDFT_ERR_UNSUPPORTED, "N1=%d must be a multiple of %d", n1, V);
  RS_CHECK(ld % 4 == 0, RSDFT_ERR_ARG, "leading dimension must keep 16-byte alignment");
  const int bx = n1 / V;
  int by = std::max(1, 256 / bx);
  by = std::min(by, (n2 + R - 1) / R);
  const int tile_y = by * R;
  const int rows = tile_y + 2 * MD;
  const int align_el = 128 / (int)sizeof(S);
  const int stage_elems = ((rows * 2 * n1 + align_el - 1) / align_el) * align_el;
  const size_t smem = (size_t)SS * stage_elems * sizeof(S) + SS * sizeof(uint64_t);
  RS_CHECK(smem <= 220 * 1024, RSDFT_ERR_UNSUPPORTED, "stencil stage (%zu B) exceeds shared memory", smem);
  const int ytiles = (n2 + tile_y - 1) / tile_y;
  int zch = 1;
  while ((long long)ytiles * zch * nb < 4 * 148 && n3 / (zch * 2) >= 16) zch *= 2;
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;
  StArgsC<S, MD> a;
  a.psi = psi; a.out = out; a.ld = (long long)ld;
  a.vloc = (std::is_same<S, double>::value ? (const S*)c.vloc64.as<double>() : (const S*)c.vloc32.as<float>()) +
           (size_t)s * c.ng;
  a.n1 = n1; a.n2 = n2; a.n3 = n3;
  a.tile_y = tile_y; a.tz = tz; a.stage_elems = stage_elems;
  a.c0 = (S)(c.p.coef_lap0 + c.kp[k].const_k2);
  for (int d = 0; d < 3; ++d)
    for (int m = 0; m < MD; ++m) {
      a.cc[d][m] = (S)c.p.coef_lap[d][m];
      a.cs[d][m] = (S)c.kp[k].coef_nabk[d][m];
    }
  const bool nl_on = c.nl.nproj > 0 && coef != nullptr;
  a.rowptr = nl_on ? c.nl.rec_rowptr.as<int>() : nullptr;
  a.rec_g = nl_on ? c.nl.rec_g.as<int>() : nullptr;
  a.val = nl_on ? (std::is_same<S, double>::value ? (const S*)c.nl.perk[k].ru64.as<double>()
                                                  : (const S*)c.nl.perk[k].ru32.as<float>())
                : nullptr;
  a.pg = c.nl.pg;
  a.coef = coef;
  a.ldc = c.nl.ngroups * c.nl.pg;
  a.status = c.d_status;
  auto kern = k_stencil_cplx<S, MD, R, SS>;
  static bool attr_done = false;
  if (!attr_done) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    attr_done = true;
  }
  const double alg_bytes = (double)sizeof(S) * (4.0 * (double)c.ng * nb + (double)c.ng) +
                           (nl_on ? 4.0 * (double)(c.ng + 1) + (8.0 + 2 * sizeof(S) * c.nl.pg) * c.nl.nrec : 0.0);
  ProfScope ps(c, "hpsi_stencil", alg_bytes);
  kern<<<dim3(ytiles, zch, nb), dim3(bx, by), smem, c.stream>>>(a);
  c.launches++;
  return check_launch("hpsi_stencil_cplx");
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
  if (c.p.md == 6) return launch_stencil_c<S, 6>(c, k, s, psi, out, ld, nb, coef);
  if (c.p.md == 4) return launch_stencil_c<S, 4>(c, k, s, psi, out, ld, nb, coef);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}
template int hpsi_cplx<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_cplx<double>(Ctx&, int, int, const double*, double*, size_t, int);

}  // namespace rsdft
