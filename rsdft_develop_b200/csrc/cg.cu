// Batched band-by-band preconditioned CG (real8 build) and the hprsdft preconditioner.
//
// Reference: d_conjugate_gradient_1 (src/conjugate_gradient/cg_module.f90:112-431) with
// MB_d = 1: every band runs its own CG independently, so all bands of a block are advanced
// together here with per-band state (E, E1, rb, gkgk, res, active flag) kept on the device.
// A band that leaves the reference's icg loop early (|E-E1| < 1e-15, which follows a
// rejected step, :233) is masked out for the rest of the call, which reproduces the
// per-band exits of MB_d = 1 exactly.  precond_hprsdft
// (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270) is batched the same way.
//
// Reductions are deterministic: each CTA writes a per-band partial sum and the scalar
// kernels add the partials of a band in a fixed order.
#include <cstring>

#include "ctx.cuh"

namespace rsdft {

constexpr int kThreads = 256;
constexpr int kMaxChunks = 128;

enum Scal {
  S_E = 0, S_E1, S_RB, S_GKGK, S_RES, S_W, S_U1, S_U2, S_ACT, S_BETA, S_ACC,
  S_RR0, S_RR1, S_PCA, S_PCB, S_PCACT, S_COUNT
};

struct Blk {
  int nbb;        // bands in the block
  int nch;        // CTAs (chunks) per band for elementwise/reduction kernels
  size_t ng;
  double* sc;     // scalars [S_COUNT][nbb]
  double* part;   // partials [nbb][nch][6]
};

__device__ __forceinline__ double& SC(const Blk& k, int which, int b) { return k.sc[(size_t)which * k.nbb + b]; }

template <int ND>
__device__ __forceinline__ void block_partials(double (&v)[ND], const Blk& k, int b) {
  __shared__ double red[kThreads / 32][ND];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    double x = v[d];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[wid][d] = x;
  }
  __syncthreads();
  if (threadIdx.x < ND) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) t += red[w][threadIdx.x];
    k.part[((size_t)b * k.nch + blockIdx.x) * 6 + threadIdx.x] = t;
  }
}

__device__ __forceinline__ double sum_part(const Blk& k, int b, int d) {
  double t = 0.0;
  for (int c = 0; c < k.nch; ++c) t += k.part[((size_t)b * k.nch + c) * 6 + d];
  return t;
}

#define BAND_LOOP(k)                                                        \
  const int b = blockIdx.y;                                                 \
  const size_t off = (size_t)b * (k).ng;                                    \
  const size_t per = ((k).ng + (k).nch - 1) / (k).nch;                      \
  const size_t i0 = per * blockIdx.x, i1 = min((k).ng, i0 + per);

// ---------------------------------------------------------------------------
// elementwise + reduction kernels
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dot(Blk k, const T* __restrict__ a, const T* __restrict__ bb,
                                                  int act_idx) {
  BAND_LOOP(k);
  if (act_idx >= 0 && SC(k, act_idx, b) == 0.0) return;
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) v[0] += (double)a[off + i] * (double)bb[off + i];
  block_partials<1>(v, k, b);
}

// g = gfac (hx - E x); partial |g|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_make_g(Blk k, const T* __restrict__ x, const T* __restrict__ hx,
                                                     T* __restrict__ g, double gfac) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  const double E = SC(k, S_E, b);
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const T gi = (T)(gfac * ((double)hx[off + i] - E * (double)x[off + i]));
    g[off + i] = gi;
    v[0] += (double)gi * (double)gi;
  }
  block_partials<1>(v, k, b);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_copy(Blk k, const T* __restrict__ src, T* __restrict__ dst) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) dst[off + i] = src[off + i];
}

// p = Pg + beta p
template <typename T>
__global__ void __launch_bounds__(kThreads) k_make_p(Blk k, const T* __restrict__ pg, T* __restrict__ p, int first) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  const T beta = (T)SC(k, S_BETA, b);
  if (first) {
    for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) p[off + i] = pg[off + i];
  } else {
    for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) p[off + i] = pg[off + i] + beta * p[off + i];
  }
}

// the six dot products of the line minimisation (cg_module.f90:288-296)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dots6(Blk k, const T* __restrict__ x, const T* __restrict__ p,
                                                    const T* __restrict__ hx, const T* __restrict__ hp) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double xi = x[off + i], pi = p[off + i], hxi = hx[off + i], hpi = hp[off + i];
    v[0] += xi * xi;
    v[1] += pi * xi;
    v[2] += pi * pi;
    v[3] += xi * hxi;
    v[4] += pi * hxi;
    v[5] += pi * hpi;
  }
  block_partials<6>(v, k, b);
}

// hx = u1 hx + u2 hp ; g = gfac (hx - W (u1 x + u2 p)) ; partial |g|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_hg(Blk k, const T* __restrict__ x, const T* __restrict__ p,
                                                        T* __restrict__ hx, const T* __restrict__ hp,
                                                        T* __restrict__ g, double gfac) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  const double u1 = SC(k, S_U1, b), u2 = SC(k, S_U2, b), W = SC(k, S_W, b);
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double h = u1 * (double)hx[off + i] + u2 * (double)hp[off + i];
    const T ht = (T)h;
    hx[off + i] = ht;
    const T gi = (T)(gfac * ((double)ht - W * (u1 * (double)x[off + i] + u2 * (double)p[off + i])));
    g[off + i] = gi;
    v[0] += (double)gi * (double)gi;
  }
  block_partials<1>(v, k, b);
}

// x = u1 x + u2 p for accepted bands
template <typename T>
__global__ void __launch_bounds__(kThreads) k_update_x(Blk k, T* __restrict__ x, const T* __restrict__ p) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0 || SC(k, S_ACC, b) == 0.0) return;
  const double u1 = SC(k, S_U1, b), u2 = SC(k, S_U2, b);
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads)
    x[off + i] = (T)(u1 * (double)x[off + i] + u2 * (double)p[off + i]);
}

// ---------------------------------------------------------------------------
// per-band scalar kernels (one thread per band)
// ---------------------------------------------------------------------------
__global__ void k_sc_init(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  SC(k, S_E, b) = sum_part(k, b, 0) * dV;
  SC(k, S_E1, b) = 1.0e10;
  SC(k, S_ACT, b) = 1.0;
  SC(k, S_RES, b) = 0.0;
}

// rb = dV * sum
__global__ void k_sc_rb(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  SC(k, S_RB, b) = sum_part(k, b, 0) * dV;
}

// loop head: res = rb / c1^2, exit tests (cg_module.f90:231-237)
__global__ void k_sc_top(Blk k, double c1sq) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = SC(k, S_RB, b);
  SC(k, S_RES, b) = rb / c1sq;
  if (rb < 0.0 || fabs(SC(k, S_E, b) - SC(k, S_E1, b)) < 1.0e-15) SC(k, S_ACT, b) = 0.0;
}

// rb = <Pg|g> dV ; beta = rb / gkgk ; gkgk = rb
__global__ void k_sc_beta(Blk k, double dV, int first) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = sum_part(k, b, 0) * dV;
  SC(k, S_RB, b) = rb;
  SC(k, S_BETA, b) = first ? 0.0 : rb / SC(k, S_GKGK, b);
  SC(k, S_GKGK, b) = rb;
}

// 2x2 generalised symmetric eigenproblem A z = w B z (dsygv itype 1, cg_module.f90:316),
// root selection (:317-321) and sign fix (:322-327).
__global__ void k_sc_solve2(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double B11 = sum_part(k, b, 0) * dV, B12 = sum_part(k, b, 1) * dV, B22 = sum_part(k, b, 2) * dV;
  const double A11 = sum_part(k, b, 3) * dV, A12 = sum_part(k, b, 4) * dV, A22 = sum_part(k, b, 5) * dV;
  const double E = SC(k, S_E, b);
  double w1, w2, z1[2], z2[2];
  bool ok = B11 > 0.0;
  double u11 = 0, u12 = 0, u22 = 0;
  if (ok) {
    u11 = sqrt(B11);
    u12 = B12 / u11;
    const double t = B22 - u12 * u12;
    ok = t > 0.0;
    if (ok) u22 = sqrt(t);
  }
  if (!ok) {
    // B not positive definite: keep the band unchanged
    SC(k, S_U1, b) = 1.0;
    SC(k, S_U2, b) = 0.0;
    SC(k, S_W, b) = E;
    SC(k, S_E1, b) = E;
    return;
  }
  // C = U^-T A U^-1
  const double l11 = 1.0 / u11, l21 = -u12 / (u11 * u22), l22 = 1.0 / u22;
  const double a = l11 * l11 * A11;
  const double c12 = l11 * (l21 * A11 + l22 * A12);
  const double d = l21 * l21 * A11 + 2.0 * l21 * l22 * A12 + l22 * l22 * A22;
  const double mean = 0.5 * (a + d), r = hypot(0.5 * (a - d), c12);
  w1 = mean - r;
  w2 = mean + r;
  double v1, v2;
  if (r == 0.0) {
    v1 = 1.0; v2 = 0.0;
  } else if (d - w1 >= a - w1) {
    v1 = d - w1; v2 = -c12;
  } else {
    v1 = c12; v2 = w1 - a;
  }
  const double nv = hypot(v1, v2);
  v1 /= nv; v2 /= nv;
  // second eigenvector (-v2, v1); back-transform z = U^-1 v
  z1[0] = v1 / u11 - u12 * v2 / (u11 * u22);
  z1[1] = v2 / u22;
  z2[0] = -v2 / u11 - u12 * v1 / (u11 * u22);
  z2[1] = v1 / u22;
  double W = w1, x1 = z1[0], x2 = z1[1];
  if (fabs(w1 - E) > 1.0e-1 && fabs(w2 - E) <= 1.0e-1) {
    W = w2; x1 = z2[0]; x2 = z2[1];
  }
  if (x1 < 0.0) { x1 = -x1; x2 = -x2; }
  SC(k, S_U1, b) = x1;
  SC(k, S_U2, b) = x2;
  SC(k, S_W, b) = W;
  SC(k, S_E1, b) = E;
  SC(k, S_E, b) = W;
}

// residual growth guard (cg_module.f90:360-363)
__global__ void k_sc_reject(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = sum_part(k, b, 0) * dV;
  SC(k, S_RB, b) = rb;
  if (rb / SC(k, S_RES, b) > 1.0e8) {
    SC(k, S_E, b) = SC(k, S_E1, b);
    SC(k, S_ACC, b) = 0.0;
  } else {
    SC(k, S_ACC, b) = 1.0;
  }
}

// ---------------------------------------------------------------------------
// preconditioner: 7-point operator A = (c0 - E0) I + sum_d c_d (shift_+ + shift_-), E0 = 0
// ---------------------------------------------------------------------------
struct PcCoef {
  double c0, c1, c2, c3;
  int n1, n2, n3;
};

template <typename T>
__device__ __forceinline__ double apply7(const T* __restrict__ g, size_t i, const PcCoef& q) {
  const int n1 = q.n1, n2 = q.n2, n3 = q.n3;
  const int i1 = (int)(i % n1);
  const int i2 = (int)((i / n1) % n2);
  const int i3 = (int)(i / ((size_t)n1 * n2));
  const size_t row = i - i1;
  const size_t pln = (size_t)n1 * n2;
  const size_t xm = row + (i1 == 0 ? n1 - 1 : i1 - 1), xp = row + (i1 == n1 - 1 ? 0 : i1 + 1);
  const size_t ym = i + (i2 == 0 ? (size_t)(n2 - 1) * n1 : 0) - (i2 == 0 ? 0 : n1);
  const size_t yp = i - (i2 == n2 - 1 ? (size_t)(n2 - 1) * n1 : 0) + (i2 == n2 - 1 ? 0 : n1);
  const size_t zm = i + (i3 == 0 ? (size_t)(n3 - 1) * pln : 0) - (i3 == 0 ? 0 : pln);
  const size_t zp = i - (i3 == n3 - 1 ? (size_t)(n3 - 1) * pln : 0) + (i3 == n3 - 1 ? 0 : pln);
  return q.c0 * (double)g[i] + q.c1 * ((double)g[xp] + (double)g[xm]) + q.c2 * ((double)g[yp] + (double)g[ym]) +
         q.c3 * ((double)g[zp] + (double)g[zm]);
}

// F = A G ; R = G - F ; Q = R ; PG = G ; partial |R|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_first(Blk k, PcCoef q, const T* __restrict__ G,
                                                       T* __restrict__ R, T* __restrict__ Q, T* __restrict__ PG) {
  BAND_LOOP(k);
  if (SC(k, S_ACT, b) == 0.0) return;
  const T* g = G + off;
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double f = apply7(g, i, q);
    const T r = (T)((double)g[i] - f);
    R[off + i] = r;
    Q[off + i] = r;
    PG[off + i] = g[i];
    v[0] += (double)r * (double)r;
  }
  block_partials<1>(v, k, b);
}

// F = A Q ; partial <Q|F>
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_apply(Blk k, PcCoef q, const T* __restrict__ Q, T* __restrict__ F) {
  BAND_LOOP(k);
  if (SC(k, S_PCACT, b) == 0.0) return;
  const T* qq = Q + off;
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double f = apply7(qq, i, q);
    F[off + i] = (T)f;
    v[0] += (double)qq[i] * (double)(T)f;
  }
  block_partials<1>(v, k, b);
}

// PG += a Q ; (if !last) R -= a F ; partial |R|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_update(Blk k, const T* __restrict__ Q, const T* __restrict__ F,
                                                        T* __restrict__ R, T* __restrict__ PG, int last) {
  BAND_LOOP(k);
  if (SC(k, S_PCACT, b) == 0.0) return;
  const double a = SC(k, S_PCA, b);
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double qi = Q[off + i];
    PG[off + i] = (T)((double)PG[off + i] + a * qi);
    if (!last) {
      const T r = (T)((double)R[off + i] - a * (double)F[off + i]);
      R[off + i] = r;
      v[0] += (double)r * (double)r;
    }
  }
  if (!last) block_partials<1>(v, k, b);
}

// Q = R + b Q
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_newdir(Blk k, const T* __restrict__ R, T* __restrict__ Q) {
  BAND_LOOP(k);
  if (SC(k, S_PCACT, b) == 0.0) return;
  const double bb = SC(k, S_PCB, b);
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) Q[off + i] = (T)((double)R[off + i] + bb * (double)Q[off + i]);
}

__global__ void k_pc_sc_first(Blk k) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  if (SC(k, S_ACT, b) == 0.0) { SC(k, S_PCACT, b) = 0.0; return; }
  const double rr1 = sum_part(k, b, 0);
  SC(k, S_RR1, b) = rr1;
  SC(k, S_PCACT, b) = rr1 < 1.0e-24 ? 0.0 : 1.0;   // cgpc_hprsdft_module.f90:181
}
__global__ void k_pc_sc_alpha(Blk k) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_PCACT, b) == 0.0) return;
  const double pAp = sum_part(k, b, 0);
  SC(k, S_RR0, b) = SC(k, S_RR1, b);
  SC(k, S_PCA, b) = SC(k, S_RR0, b) / pAp;
}
__global__ void k_pc_sc_beta(Blk k) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_PCACT, b) == 0.0) return;
  const double rr1 = sum_part(k, b, 0);
  SC(k, S_RR1, b) = rr1;
  SC(k, S_PCB, b) = rr1 / SC(k, S_RR0, b);
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
static int pick_nch(size_t ng, int nbb) {
  int nch = (int)std::min<size_t>(kMaxChunks, (ng + 4095) / 4096);
  while (nch > 1 && (long long)nch * nbb > 16 * 148 * 4) nch /= 2;
  return std::max(1, nch);
}

#define LAUNCH_E(kern, ...)                                                  \
  do {                                                                       \
    kern<<<dim3(k.nch, k.nbb), kThreads, 0, c.stream>>>(k, __VA_ARGS__);     \
    c.launches++;                                                            \
  } while (0)
#define LAUNCH_S(kern, ...)                                                  \
  do {                                                                       \
    kern<<<(k.nbb + 127) / 128, 128, 0, c.stream>>>(k, ##__VA_ARGS__);       \
    c.launches++;                                                            \
  } while (0)

template <typename T>
static int pc_block(Ctx& c, Blk& k, const T* G, T* PG, T* R, T* Q, T* F) {
  PcCoef q;
  const double* H = c.p.hgrid;
  q.c0 = c.p.ggg[0] / (H[0] * H[0]) + c.p.ggg[1] / (H[1] * H[1]) + c.p.ggg[2] / (H[2] * H[2]);
  q.c1 = -0.5 * c.p.ggg[0] / (H[0] * H[0]);
  q.c2 = -0.5 * c.p.ggg[1] / (H[1] * H[1]);
  q.c3 = -0.5 * c.p.ggg[2] / (H[2] * H[2]);
  q.n1 = c.p.n1; q.n2 = c.p.n2; q.n3 = c.p.n3;
  ProfScope ps(c, "pc");
  LAUNCH_E(k_pc_first<T>, q, G, R, Q, PG);
  LAUNCH_S(k_pc_sc_first);
  for (int it = 1; it <= c.p.mloop; ++it) {
    LAUNCH_E(k_pc_apply<T>, q, Q, F);
    LAUNCH_S(k_pc_sc_alpha);
    const int last = it == c.p.mloop;
    LAUNCH_E(k_pc_update<T>, Q, F, R, PG, last);
    if (last) break;
    LAUNCH_S(k_pc_sc_beta);
    LAUNCH_E(k_pc_newdir<T>, R, Q);
  }
  return check_launch("pc");
}

template <typename T>
int precond_real(Ctx& c, const T* g, T* pg, size_t ld, int nb) {
  RS_CHECK(ld == c.ng, RSDFT_ERR_ARG, "precond: ld must equal the grid size");
  Blk k;
  k.nbb = nb;
  k.ng = c.ng;
  k.nch = pick_nch(c.ng, nb);
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nb + 64));
  RS_TRY(c.ws_red.ensure(sizeof(double) * 6 * (size_t)nb * k.nch));
  RS_TRY(c.ws_cg.ensure(sizeof(T) * 3 * c.ng * (size_t)nb));
  k.sc = c.ws_scal.as<double>();
  k.part = c.ws_red.as<double>();
  std::vector<double> act((size_t)nb, 1.0);
  RS_CUDA(cudaMemcpyAsync(k.sc + (size_t)S_ACT * nb, act.data(), sizeof(double) * nb, cudaMemcpyHostToDevice,
                          c.stream));
  T* R = c.ws_cg.as<T>();
  T* Q = R + c.ng * nb;
  T* F = Q + c.ng * nb;
  RS_TRY(pc_block<T>(c, k, g, pg, R, Q, F));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}
template int precond_real<double>(Ctx&, const double*, double*, size_t, int);
template int precond_real<float>(Ctx&, const float*, float*, size_t, int);

template <typename T>
static int cg_real(Ctx& c, int kk, int s, double* h_esp, double* h_res) {
  const int nb = c.kp[kk].nband;
  const size_t ng = c.ng;
  int nbb = c.p.cg_block > 0 ? std::min(c.p.cg_block, nb) : nb;
  // budget: 8 block vectors per band; keep them within ~40% of free memory
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  const size_t per_band = 8 * ng * sizeof(T);
  const size_t have = c.ws_cg.bytes;
  const size_t budget = (size_t)(0.4 * (double)(freeb + have));
  if (c.p.cg_block <= 0) {
    while (nbb > 1 && (size_t)nbb * per_band > budget) nbb = (nbb + 1) / 2;
  }
  RS_TRY(c.ws_cg.ensure(per_band * nbb));
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nbb + 64));
  Blk k;
  k.nbb = nbb;
  k.ng = ng;
  k.nch = pick_nch(ng, nbb);
  RS_TRY(c.ws_red.ensure(sizeof(double) * 6 * (size_t)nbb * k.nch));
  k.sc = c.ws_scal.as<double>();
  k.part = c.ws_red.as<double>();
  T* base = c.ws_cg.as<T>();
  T* HX = base;
  T* HP = HX + ng * nbb;
  T* G = HP + ng * nbb;
  T* PG = G + ng * nbb;
  T* P = PG + ng * nbb;
  T* R = P + ng * nbb;
  T* Q = R + ng * nbb;
  T* F = Q + ng * nbb;
  T* psi = c.wfn(kk, s).psi.as<T>();
  const double dV = c.p.dv;
  const double gfac = -2.0, c1sq = 4.0;  // real build: g = -2(Hx - Ex), res = rb / 2^2
  std::vector<double> hE, hR;
  for (int b0 = 0; b0 < nb; b0 += nbb) {
    const int nn = std::min(nbb, nb - b0);
    k.nbb = nn;
    k.nch = pick_nch(ng, nn);
    T* X = psi + (size_t)b0 * ng;
    {
      ProfScope ps(c, "cg");
      RS_TRY(hpsi_real<T>(c, kk, s, X, HX, ng, nn));
    }
    {
      ProfScope ps(c, "cg");
      LAUNCH_E(k_dot<T>, X, HX, -1);
      LAUNCH_S(k_sc_init, dV);
      LAUNCH_E(k_make_g<T>, X, HX, G, gfac);
      LAUNCH_S(k_sc_rb, dV);
    }
    for (int icg = 1; icg <= c.p.ncg + 1; ++icg) {
      {
        ProfScope ps(c, "cg");
        LAUNCH_S(k_sc_top, c1sq);
      }
      if (icg == c.p.ncg + 1) break;
      if (c.p.pc_mode == RSDFT_PC_NONE) {
        ProfScope ps(c, "cg");
        LAUNCH_E(k_copy<T>, G, PG);
      } else {
        RS_TRY(pc_block<T>(c, k, G, PG, R, Q, F));
      }
      {
        ProfScope ps(c, "cg");
        LAUNCH_E(k_dot<T>, PG, G, (int)S_ACT);
        LAUNCH_S(k_sc_beta, dV, icg == 1 ? 1 : 0);
        LAUNCH_E(k_make_p<T>, PG, P, icg == 1 ? 1 : 0);
      }
      RS_TRY(hpsi_real<T>(c, kk, s, P, HP, ng, nn));
      {
        ProfScope ps(c, "cg");
        LAUNCH_E(k_dots6<T>, X, P, HX, HP);
        LAUNCH_S(k_sc_solve2, dV);
        LAUNCH_E(k_update_hg<T>, X, P, HX, HP, G, gfac);
        LAUNCH_S(k_sc_reject, dV);
        LAUNCH_E(k_update_x<T>, X, P);
      }
    }
    RS_TRY(check_launch("cg"));
    if (h_esp || h_res) {
      hE.resize(nn);
      hR.resize(nn);
      RS_CUDA(cudaMemcpyAsync(hE.data(), k.sc + (size_t)S_E * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost, c.stream));
      RS_CUDA(cudaMemcpyAsync(hR.data(), k.sc + (size_t)S_RES * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost,
                              c.stream));
      RS_CUDA(cudaStreamSynchronize(c.stream));
      if (h_esp) std::memcpy(h_esp + b0, hE.data(), sizeof(double) * nn);
      if (h_res) std::memcpy(h_res + b0, hR.data(), sizeof(double) * nn);
    }
  }
  return 0;
}

int cg_run(Ctx& c, int k, int s, double* h_esp, double* h_res) {
  if (c.cplx) {
    RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "complex16 CG is provided by cg_cplx");
  }
  if (c.mixed) return cg_real<float>(c, k, s, h_esp, h_res);
  return cg_real<double>(c, k, s, h_esp, h_res);
}

}  // namespace rsdft

namespace rsdft {

// ---------------------------------------------------------------------------
// FP64 residual check (esp_calc + the CG residual definition, in FP64 for any storage)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_res_dots(Blk k, const T* __restrict__ x, const double* __restrict__ hx) {
  BAND_LOOP(k);
  double v[2] = {0.0, 0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double xi = (double)x[off + i];
    v[0] += xi * xi;
    v[1] += xi * hx[off + i];
  }
  block_partials<2>(v, k, b);
}
__global__ void k_res_sc1(Blk k, double* esp) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  const double xx = sum_part(k, b, 0), xh = sum_part(k, b, 1);
  SC(k, S_RR0, b) = xx;
  SC(k, S_E, b) = xh / xx;
  esp[b] = xh / xx;
}
template <typename T>
__global__ void __launch_bounds__(kThreads) k_res_norm(Blk k, const T* __restrict__ x, const double* __restrict__ hx) {
  BAND_LOOP(k);
  const double e = SC(k, S_E, b);
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double r = hx[off + i] - e * (double)x[off + i];
    v[0] += r * r;
  }
  block_partials<1>(v, k, b);
}
__global__ void k_res_sc2(Blk k, double* res) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  res[b] = sum_part(k, b, 0) / SC(k, S_RR0, b);
}

template <typename T>
static int residual_real(Ctx& c, int kk, int s, double* d_esp, double* d_res) {
  const int nb = c.kp[kk].nband;
  const size_t ng = c.ng;
  // band chunk so that the FP64 copies stay around 1 GiB
  int nbc = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)(1u << 30) / (16 * ng)));
  const size_t extra = std::is_same<T, double>::value ? 0 : 1;
  RS_TRY(c.ws_rot.ensure(sizeof(double) * ng * nbc * (1 + extra)));
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nbc + sizeof(double) * 2 * nb + 64));
  const T* psi = c.wfn(kk, s).psi.as<T>();
  double* HX = c.ws_rot.as<double>();
  double* XD = HX + ng * nbc;
  Blk k;
  k.ng = ng;
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int nn = std::min(nbc, nb - b0);
    k.nbb = nn;
    k.nch = pick_nch(ng, nn);
    RS_TRY(c.ws_red.ensure(sizeof(double) * 6 * (size_t)nn * k.nch));
    k.sc = c.ws_scal.as<double>();
    k.part = c.ws_red.as<double>();
    const T* X = psi + (size_t)b0 * ng;
    const double* XH;
    if (std::is_same<T, double>::value) {
      XH = reinterpret_cast<const double*>(X);
    } else {
      RS_TRY(convert_f2d(c, reinterpret_cast<const float*>(X), XD, ng * nn));
      XH = XD;
    }
    RS_TRY(hpsi_real<double>(c, kk, s, XH, HX, ng, nn));
    ProfScope ps(c, "residual");
    LAUNCH_E(k_res_dots<T>, X, HX);
    LAUNCH_S(k_res_sc1, d_esp + b0);
    LAUNCH_E(k_res_norm<T>, X, HX);
    LAUNCH_S(k_res_sc2, d_res + b0);
  }
  return check_launch("residual");
}

int residual_run(Ctx& c, int k, int s, double* d_esp, double* d_res) {
  RS_CHECK(!c.cplx, RSDFT_ERR_UNSUPPORTED, "complex16 residual is provided by residual_cplx");
  if (c.mixed) return residual_real<float>(c, k, s, d_esp, d_res);
  return residual_real<double>(c, k, s, d_esp, d_res);
}

}  // namespace rsdft
