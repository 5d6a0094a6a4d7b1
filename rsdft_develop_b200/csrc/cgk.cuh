// Per-band state of the batched CG and its preconditioner, shared by cg.cu (the CG step and the
// multi-pass preconditioner) and pc_stream.cu (the fused z-streamed preconditioner).
//
// Every band of a block carries its scalars (E, E1, rb, ... as cg_module.f90 keeps them per band)
// in one device array [S_COUNT][nbb]; reductions leave per-CTA partial sums in [nbb][nch][kPS],
// which the one-thread-per-band scalar kernels add in a fixed order (deterministic).
#pragma once
#include "ctx.cuh"

namespace rsdft {

constexpr int kThreads = 256;
constexpr int kMaxChunks = 128;
constexpr int kPS = 16;  // partial slots per (band, chunk)

enum Scal {
  S_E = 0, S_E1, S_RB, S_GKGK, S_RES, S_W, S_U1, S_U1I, S_U2, S_U2I, S_ACT, S_BETA, S_ACC,
  S_RR0, S_RR1, S_PCA, S_PCB, S_PCACT,
  S_DEF,                     // real build: x update deferred until the exact reject test (1) or done with H x (0)
  S_MU0, S_MU7 = S_MU0 + 7,  // s-step preconditioner: moments <v0 | B^i v0>, i < 2 mloop
  S_XI0, S_XI3 = S_XI0 + 3,  // s-step preconditioner: PG = G + sum_i xi_i B^i v0
  S_NU0, S_NU1,              // s-step preconditioner: <v0 | G>, <B v0 | G> (for <PG | G> without a pass)
  S_COUNT
};

struct Blk {
  int nbb;        // bands in the block
  int nch;        // CTAs (chunks) per band for elementwise/reduction kernels
  size_t ng;      // reals per band (grid points x components)
  double* sc;     // scalars [S_COUNT][nbb]
  double* part;   // partials [nbb][nch][kPS]
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
    k.part[((size_t)b * k.nch + blockIdx.x) * kPS + threadIdx.x] = t;
  }
}

__device__ __forceinline__ double sum_part(const Blk& k, int b, int d) {
  double t = 0.0;
  for (int c = 0; c < k.nch; ++c) t += k.part[((size_t)b * k.nch + c) * kPS + d];
  return t;
}

// The mloop CG steps of precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:189-260)
// on coefficient vectors in the Krylov basis v_i = B^i r0 (A = c0 (B + I)), every inner product
// taken from the moments mu_j = <r0 | B^j r0>, j < 2m: leaves PG = G + sum_{i<m} xi_i v_i.
__device__ __forceinline__ void pcs_recurrence(const double* mu, int m, double c0, double* xi) {
  double p[5] = {1.0, 0.0, 0.0, 0.0, 0.0}, r[5] = {1.0, 0.0, 0.0, 0.0, 0.0}, f[5];
  for (int j = 0; j < 5; ++j) xi[j] = 0.0;
  double rr1 = mu[0], rr0;
  for (int it = 1; it <= m; ++it) {
    // f = A p = c0 (B p + p); p has degree it - 1, f degree it
    for (int j = 0; j <= it; ++j) f[j] = c0 * ((j > 0 ? p[j - 1] : 0.0) + (j < it ? p[j] : 0.0));
    double pAp = 0.0;
    for (int a = 0; a < it; ++a)
      for (int c = 0; c <= it; ++c) pAp += p[a] * f[c] * mu[a + c];
    rr0 = rr1;
    const double al = rr0 / pAp;
    for (int j = 0; j < it; ++j) xi[j] += al * p[j];
    if (it == m) break;
    for (int j = 0; j <= it; ++j) r[j] -= al * f[j];
    rr1 = 0.0;
    for (int a = 0; a <= it; ++a)
      for (int c = 0; c <= it; ++c) rr1 += r[a] * r[c] * mu[a + c];
    const double be = rr1 / rr0;
    for (int j = 0; j <= it; ++j) p[j] = r[j] + be * p[j];
  }
}

// Fused, z-streamed form of the FP32 s-step preconditioner followed by the CG direction update
// p = PG + beta p (pc_stream.cu).  Applicable to FP32 bands with mloop 1..3; returns
// RSDFT_ERR_UNSUPPORTED (without launching anything) where it does not apply.
bool pc_fused_applies(const Ctx& c);
int pc_fused_step(Ctx& c, Blk& k, const float* G, float* P, int first);
// partial-buffer size (doubles) the fused form needs for a block of nbb bands
size_t pc_fused_part_doubles(const Ctx& c, int nbb);

}  // namespace rsdft
