// Many-band hpsi for the real8 (Gamma) build: H psi = T psi + Vloc psi + V_NL psi.
//
// Reference semantics (restated, not translated):
//   kinetic + Vloc  src/kinetic/d_kinetic_sol_module.f90:244-292  (Md=6 star stencil,
//                   (coef_lap0 + Vloc) on the centre, periodic halo src/bc/bcset_3_module.f90)
//   nonlocal        src/ps_nloc_mr_module.f90:1159-1258 (gather uVunk = dV sum uVk psi(JJP),
//                   Dij pairs, scatter psi(JJP) += uVk * sum Dij uVunk); the KB form
//                   src/d_ps_nloc2_op_module.f90:146-288 is the diagonal-Dij case.
//
// Design (B200): one pass over psi per band.  A CTA owns an (N1 x TY) column of the
// grid for one band and streams it along z.  Each xy-plane of the column (with a
// Md-deep y halo, periodic rows wrapped) is staged into shared memory by the bulk-copy
// (TMA) engine through an S-deep mbarrier ring; x taps wrap inside the staged row (the
// CTA holds full rows), y taps read neighbouring staged rows, and z taps are applied
// "push" style into 2*Md+1 rotating register accumulators, so no plane is read twice
// from memory.  The finished plane gets V_loc and the nonlocal scatter (a per-point
// CSR over the projector footprints) before one vector store.  The projector gather
// + Dij runs before, in an atom-centred kernel.
#include "ctx.cuh"
#include "ptx.cuh"

namespace rsdft {

template <typename T> struct VecT;
template <> struct VecT<float> { static constexpr int V = 4; using type = float4; };
template <> struct VecT<double> { static constexpr int V = 2; using type = double2; };

template <typename T, int V>
__device__ __forceinline__ void ldv(const T* p, T (&v)[V]) {
  using VT = typename VecT<T>::type;
  VT t = *reinterpret_cast<const VT*>(p);
  const T* tt = reinterpret_cast<const T*>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) v[i] = tt[i];
}
template <typename T, int V>
__device__ __forceinline__ void ldv_g(const T* p, T (&v)[V]) {
  using VT = typename VecT<T>::type;
  VT t = __ldg(reinterpret_cast<const VT*>(p));
  const T* tt = reinterpret_cast<const T*>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) v[i] = tt[i];
}
template <typename T, int V>
__device__ __forceinline__ void stv(T* p, const T (&v)[V]) {
  using VT = typename VecT<T>::type;
  VT t;
  T* tt = reinterpret_cast<T*>(&t);
#pragma unroll
  for (int i = 0; i < V; ++i) tt[i] = v[i];
  *reinterpret_cast<VT*>(p) = t;
}

__device__ __forceinline__ int pmod(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

template <typename T, int MD>
struct StArgs {
  const T* psi;
  T* out;
  long long ld;
  const T* vloc;
  int n1, n2, n3;
  int tile_y, tz, stage_elems;
  T c0;
  T cx[MD], cy[MD], cz[MD];
  const int* rowptr;
  const int* col;
  const T* val;
  const T* coef;
  int ldc;
  unsigned* status;
};

constexpr uint32_t kWaitPolls = 1u << 22;

template <typename T, int MD, int R, int S>
__global__ void __launch_bounds__(256) k_stencil_real(const StArgs<T, MD> a) {
  constexpr int V = VecT<T>::V;
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + V - 1) / V;
  extern __shared__ __align__(128) unsigned char smem[];
  T* stages = reinterpret_cast<T*>(smem);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + (size_t)S * a.stage_elems * sizeof(T));

  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const int x0 = threadIdx.x * V;
  const int yl = threadIdx.y * R;
  const int y0 = blockIdx.x * a.tile_y;
  const int z0 = blockIdx.y * a.tz;
  const int zend = min(z0 + a.tz, n3);
  const int rows = a.tile_y + 2 * MD;
  const int nplanes = (zend - z0) + 2 * MD;
  const T* src = a.psi + (long long)blockIdx.z * a.ld;
  T* dst = a.out + (long long)blockIdx.z * a.ld;
  const T* coefb = a.coef ? a.coef + (long long)blockIdx.z * a.ldc : nullptr;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](int q) {
    const int zg = pmod(z0 - MD + q, n3);
    T* st = stages + (size_t)(q % S) * a.stage_elems;
    uint64_t* br = &bar[q % S];
    mbar_arrive_expect_tx(br, (uint32_t)((size_t)rows * n1 * sizeof(T)));
    int r = 0;
    while (r < rows) {
      const int gy = pmod(y0 - MD + r, n2);
      const int len = min(rows - r, n2 - gy);
      bulk_g2s(st + (size_t)r * n1, src + ((size_t)zg * n2 + gy) * n1,
               (uint32_t)((size_t)len * n1 * sizeof(T)), br);
      r += len;
    }
  };
  if (tid == 0) {
    for (int q = 0; q < S - 1 && q < nplanes; ++q) issue(q);
  }

  bool rowok[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rowok[r] = (y0 + yl + r) < n2;

  T acc[NQ][R][V];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < V; ++i) acc[q][r][i] = T(0);

  int issued_upto = min(S - 1, nplanes);  // planes [0, issued_upto) issued (thread 0's view)
  bool aborted = false;
  for (int qb = 0; qb < nplanes && !aborted; qb += NQ) {
#pragma unroll
    for (int s = 0; s < NQ; ++s) {
      const int q = qb + s;
      if (q < nplanes && !aborted) {
        if (tid == 0 && q + S - 1 < nplanes) {
          fence_proxy_async_smem();
          issue(q + S - 1);
          issued_upto = q + S;
        }
        bool ok = mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
        if (__syncthreads_or(!ok)) {
          aborted = true;
          if (tid == 0) atomicOr(a.status, DEV_WAIT_TIMEOUT);
          break;
        }
        const T* pl = stages + (size_t)(q % S) * a.stage_elems;
        const int p = z0 - MD + q;
        T v[R][V];
#pragma unroll
        for (int r = 0; r < R; ++r) ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + x0, v[r]);

        if (p >= z0 && p < zend) {
          T t[R][V];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            T vl[V];
            if (rowok[r]) {
              ldv_g<T, V>(a.vloc + ((size_t)p * n2 + (y0 + yl + r)) * n1 + x0, vl);
            } else {
#pragma unroll
              for (int i = 0; i < V; ++i) vl[i] = T(0);
            }
#pragma unroll
            for (int i = 0; i < V; ++i) t[r][i] = (a.c0 + vl[i]) * v[r][i];
            // x taps: full periodic row is staged; chunks wrap modulo N1
            T w[(2 * NCH + 1) * V];
#pragma unroll
            for (int i = 0; i < V; ++i) w[NCH * V + i] = v[r][i];
#pragma unroll
            for (int ch = 1; ch <= NCH; ++ch) {
              T lf[V], rt[V];
              ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + pmod(x0 - ch * V, n1), lf);
              ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + pmod(x0 + ch * V, n1), rt);
#pragma unroll
              for (int i = 0; i < V; ++i) {
                w[(NCH - ch) * V + i] = lf[i];
                w[(NCH + ch) * V + i] = rt[i];
              }
            }
#pragma unroll
            for (int i = 0; i < V; ++i)
#pragma unroll
              for (int m = 1; m <= MD; ++m)
                t[r][i] += a.cx[m - 1] * (w[NCH * V + i - m] + w[NCH * V + i + m]);
          }
          // y taps
#pragma unroll
          for (int dy = -MD; dy < R + MD; ++dy) {
            T rv[V];
            if (dy >= 0 && dy < R) {
#pragma unroll
              for (int i = 0; i < V; ++i) rv[i] = v[dy >= 0 && dy < R ? dy : 0][i];
            } else {
              ldv<T, V>(pl + (size_t)(yl + dy + MD) * n1 + x0, rv);
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int m = dy > r ? dy - r : r - dy;
              if (m >= 1 && m <= MD) {
#pragma unroll
                for (int i = 0; i < V; ++i) t[r][i] += a.cy[(m >= 1 ? m : 1) - 1] * rv[i];
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) acc[s][r][i] += t[r][i];
        }
        // z taps, pushed into the accumulators of planes p-m and p+m
#pragma unroll
        for (int m = 1; m <= MD; ++m) {
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) {
              acc[(s - m + NQ) % NQ][r][i] += a.cz[m - 1] * v[r][i];
              acc[(s + m) % NQ][r][i] += a.cz[m - 1] * v[r][i];
            }
        }
        // plane p - MD is complete
        {
          constexpr int fs_dummy = 0;
          (void)fs_dummy;
          const int zo = p - MD;
          const int fs = (s + NQ - MD) % NQ;
          if (zo >= z0 && zo < zend) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
              if (rowok[r]) {
                T o[V];
#pragma unroll
                for (int i = 0; i < V; ++i) o[i] = acc[fs][r][i];
                const size_t g = ((size_t)zo * n2 + (y0 + yl + r)) * n1 + x0;
                if (a.rowptr) {
                  const int e0 = __ldg(a.rowptr + g), eV = __ldg(a.rowptr + g + V);
                  if (e0 != eV) {
#pragma unroll
                    for (int i = 0; i < V; ++i) {
                      const int ea = __ldg(a.rowptr + g + i), eb = __ldg(a.rowptr + g + i + 1);
                      for (int e = ea; e < eb; ++e) o[i] += __ldg(a.val + e) * __ldg(coefb + __ldg(a.col + e));
                    }
                  }
                }
                stv<T, V>(dst + g, o);
              }
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r)
#pragma unroll
            for (int i = 0; i < V; ++i) acc[fs][r][i] = T(0);
        }
        __syncthreads();
      }
    }
  }
  if (aborted && tid == 0) {
    // drain copies still in flight before the CTA's shared memory is released
    for (int q = 0; q < issued_upto; ++q) mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
  }
}

// ---------------------------------------------------------------------------
// nonlocal gather + Dij (atom-centred): coef[b][lma] = sum_q D[lma][q] dV sum_j uV(j,q) psi_b(JJ(j))
// ---------------------------------------------------------------------------
template <typename T, int PG, int BB>
__global__ void __launch_bounds__(256) k_nl_gather_real(const T* __restrict__ psi, long long ld, int nb,
                                                        const int* __restrict__ gofs, const int* __restrict__ gjj,
                                                        const T* __restrict__ gw, const int* __restrict__ gplist,
                                                        const double* __restrict__ gD, double dV, T* coef,
                                                        int ldc) {
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
    const int lma = gplist[g * PG + p];
    if (lma >= 0 && b0 + bb < nb) {
      double cfs = 0.0;
#pragma unroll
      for (int q = 0; q < PG; ++q) cfs += gD[((size_t)g * PG + p) * PG + q] * u[bb * PG + q];
      coef[(long long)(b0 + bb) * ldc + lma] = (T)cfs;
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
  k_nl_gather_real<T, PG, BB><<<grid, 256, 0, c.stream>>>(psi, (long long)ld, nb, nl.gofs.as<int>(),
                                                           nl.gjj.as<int>(), gw, nl.gplist.as<int>(),
                                                           nl.gD.as<double>(), c.p.dv, coef, nl.nproj);
  c.launches++;
}

template <typename T>
static int nl_gather(Ctx& c, int k, const T* psi, size_t ld, int nb, T* coef) {
  NonlocalTables& nl = c.nl;
  const T* gw = std::is_same<T, double>::value ? nl.perk[k].gw64.as<T>() : nl.perk[k].gw32.as<T>();
  ProfScope ps(c, "nl_gather");
  switch (nl.pg) {
    case 1: launch_gather<T, 1, 8>(c, psi, ld, nb, coef, gw); break;
    case 4: launch_gather<T, 4, 8>(c, psi, ld, nb, coef, gw); break;
    case 9: launch_gather<T, 9, 4>(c, psi, ld, nb, coef, gw); break;
    case 16: launch_gather<T, 16, 2>(c, psi, ld, nb, coef, gw); break;
    default: RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "projectors per atom > 16 not built in");
  }
  return check_launch("nl_gather");
}

template <typename T, int MD>
static int launch_stencil(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef) {
  constexpr int V = VecT<T>::V;
  constexpr int R = 2;
  constexpr int S = 4;
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  RS_CHECK(n1 % V == 0 && n1 / V <= 256, RSDFT_ERR_UNSUPPORTED, "N1=%d must be a multiple of %d (<= %d)", n1, V,
           256 * V);
  RS_CHECK(ld % V == 0, RSDFT_ERR_ARG, "leading dimension must be a multiple of %d", V);
  const int bx = n1 / V;
  int by = std::max(1, 256 / bx);
  by = std::min(by, (n2 + R - 1) / R);
  const int tile_y = by * R;
  const int rows = tile_y + 2 * MD;
  const int align_el = 128 / (int)sizeof(T);
  const int stage_elems = ((rows * n1 + align_el - 1) / align_el) * align_el;
  const size_t smem = (size_t)S * stage_elems * sizeof(T) + S * sizeof(uint64_t);
  RS_CHECK(smem <= 220 * 1024, RSDFT_ERR_UNSUPPORTED, "stencil stage (%zu B) exceeds shared memory", smem);
  const int ytiles = (n2 + tile_y - 1) / tile_y;
  // z chunks: enough CTAs to fill the machine several times
  int zch = 1;
  while ((long long)ytiles * zch * nb < 4 * 148 && n3 / (zch * 2) >= 16) zch *= 2;
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;

  StArgs<T, MD> a;
  a.psi = psi;
  a.out = out;
  a.ld = (long long)ld;
  a.vloc = (std::is_same<T, double>::value ? c.vloc64.as<T>() : c.vloc32.as<T>()) + (size_t)s * c.ng;
  a.n1 = n1; a.n2 = n2; a.n3 = n3;
  a.tile_y = tile_y; a.tz = tz; a.stage_elems = stage_elems;
  a.c0 = (T)(c.p.coef_lap0 + c.kp[k].const_k2);
  for (int m = 0; m < MD; ++m) {
    a.cx[m] = (T)c.p.coef_lap[0][m];
    a.cy[m] = (T)c.p.coef_lap[1][m];
    a.cz[m] = (T)c.p.coef_lap[2][m];
  }
  const bool nl_on = c.nl.nproj > 0 && coef != nullptr;
  a.rowptr = nl_on ? c.nl.rowptr.as<int>() : nullptr;
  a.col = nl_on ? c.nl.col.as<int>() : nullptr;
  a.val = nl_on ? (std::is_same<T, double>::value ? c.nl.perk[k].val64.as<T>() : c.nl.perk[k].val32.as<T>())
                : nullptr;
  a.coef = coef;
  a.ldc = c.nl.nproj;
  a.status = c.d_status;
  auto kern = k_stencil_real<T, MD, R, S>;
  static bool attr_done = false;  // one per template instantiation
  if (!attr_done) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
    attr_done = true;
  }
  dim3 grid(ytiles, zch, nb), block(bx, by);
  // algorithmic bytes: read psi + write H psi per band, V_loc and the scatter tables once
  const double alg_bytes = (double)sizeof(T) * (2.0 * (double)c.ng * nb + (double)c.ng) +
                           (nl_on ? 4.0 * (double)(c.ng + 1) + (4.0 + sizeof(T)) * c.nl.nnz : 0.0);
  ProfScope ps(c, "hpsi_stencil", alg_bytes);
  kern<<<grid, block, smem, c.stream>>>(a);
  c.launches++;
  return check_launch("hpsi_stencil");
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
    RS_TRY(c.ws_coef.ensure((size_t)nb * c.nl.nproj * sizeof(T)));
    coef = c.ws_coef.as<T>();
    RS_TRY(nl_gather<T>(c, k, psi, ld, nb, coef));
  }
  if (c.p.md == 6) return launch_stencil<T, 6>(c, k, s, psi, out, ld, nb, coef);
  if (c.p.md == 4) return launch_stencil<T, 4>(c, k, s, psi, out, ld, nb, coef);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}

template int hpsi_real<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_real<double>(Ctx&, int, int, const double*, double*, size_t, int);

}  // namespace rsdft
