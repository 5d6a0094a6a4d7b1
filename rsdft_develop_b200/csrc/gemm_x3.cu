// Split-BF16 GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Each FP32 (or FP64) operand value x is split into three BF16 terms
//   x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1)
// and a product a*b is formed from the six leading cross terms
//   a0b0 + a0b1 + a1b0 + a0b2 + a1b1 + a2b0
// accumulated in FP32 in tensor memory (about FP32 accuracy; the dropped terms are
// O(2^-24) relative).  Split-K partial tiles are added into FP64 results.  With two terms
// (x0, x1) all four pairs are formed, (a0 + a1)(b0 + b1) exactly: each product keeps the
// values' 16-bit representation error (about 2^-17 relative, unbiased), which a contraction
// over K points averages down.
//
// Dense band-space work of the band update that runs through here in mixed precision:
//   overlap  S = dV Psi^T Psi (Gram-Schmidt, gram_schmidt_t_module.f90 / CholQR S),
//   Hsub     = dV Psi^T (H Psi)  (subspace_diag_la_module.f90:86),
//   rotation Psi <- Psi V        (subspace_diag_la_module.f90:190; GS: Psi <- Psi R^-1).
//
// Kernel structure: one CTA computes a 128 x BN output tile over a K range.  Warp 0 (one
// elected lane) streams the 2T operand planes (T terms of A and of B) of each KB-wide K block
// into shared memory with 3-D TMA tile loads (128B or 64B swizzle, zero fill past the matrix
// edge) through an S-deep mbarrier ring; warp 1 (one elected lane) issues KB/16 x (6 or 4)
// tcgen05.mma (K=16 steps x term pairs) per block into a 128 x BN FP32 accumulator in tensor
// memory and releases each
// stage with tcgen05.commit; after the last block all four warps read their 32 TMEM lanes
// with tcgen05.ld and write the tile.  Every wait is bounded: a timeout sets the device
// status word, drains, frees the tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include "ctx.cuh"
#include "ptx.cuh"

namespace rsdft {

namespace x3 {

constexpr int BM = 128;       // tile rows (TMEM lanes)
constexpr int kThreads = 128;
constexpr uint32_t kPolls = 1u << 24;

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// K-major operand tile with rows of KB bf16 (KB = 64: 128-byte rows, 128B swizzle; KB = 32:
// 64-byte rows, 64B swizzle), 8-row groups stored contiguously
template <int KB>
__device__ __forceinline__ uint64_t swz_desc(const void* tile) {
  const uint64_t addr = smem_u32(tile);
  uint64_t d = (addr >> 4) & 0x3FFFull;                  // start address
  d |= 1ull << 16;                                       // LBO = 16 B (ignored for swizzled K-major)
  d |= (uint64_t)((8 * KB * 2) >> 4) << 32;              // SBO: bytes between 8-row groups
  d |= 1ull << 46;                                       // descriptor version (sm_100)
  d |= (uint64_t)(KB == 64 ? 2 : 4) << 61;               // SWIZZLE_128B / SWIZZLE_64B
  return d;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,"
      "%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

struct Out {
  int mode;        // 0: C[m][n] += alpha * D (FP64 atomics); 1: Y[n*ldy + m] = D (FP32 store);
                   // 2: Y[n*ldy + m] += D (FP32); 3: complex interleaved store, column n = 2 j + c
                   // of row m to Y[j*ldy + 2 m + c]
  double* Cp[4];   // mode 0: columns [p nsplit, (p + 1) nsplit) go to Cp[p][m][n - p nsplit]
  int nsplit;
  int tri;         // mode 0: 1, the first part only by tiles reaching n <= m; 2, both parts
  long long ldc;
  double alpha;
  float* Y;
  long long ldy;
  int M, N;        // valid extents
};

// A: T planes of [M][K], B: T planes of [N][K], bf16, K-major, in K blocks of KB.
// grid = (mtiles, ntiles, ksplit).
template <int BN, int S, int T, int KB>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_x3(const __grid_constant__ CUtensorMap ta,
                                                        const __grid_constant__ CUtensorMap tb, int kblocks_total,
                                                        int kblocks_per_split, Out o, unsigned* status) {
  constexpr int A_BYTES = BM * KB * 2;       // one plane tile
  constexpr int B_BYTES = BN * KB * 2;
  constexpr int STAGE = T * A_BYTES + T * B_BYTES;
  constexpr int NP = T == 3 ? 6 : 4;  // term pairs formed
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte alignment of every tile (swizzle atoms)
  unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  // tri = 1: the first part (columns n < nsplit, the overlap S, whose two triangles hold the
  // same products) is formed only where it reaches n <= m: a tile wholly above the diagonal is
  // left out unless it also holds columns of the second part (formed in full).
  // tri = 2: both parts by triangle tiles.
  if (o.tri) {
    const bool s_part = n0 < o.nsplit, m_part = n0 + BN > o.nsplit;
    const bool s_above = !s_part || n0 >= m0 + BM;
    const bool m_above = !m_part || (o.tri == 2 && max(n0 - o.nsplit, 0) >= m0 + BM);
    if (s_above && m_above) return;
  }
  const int kb0 = blockIdx.z * kblocks_per_split;
  const int kb1 = min(kblocks_total, kb0 + kblocks_per_split);
  const int nkb = kb1 - kb0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 0) {  // allocate BN columns of tensor memory (power of two >= 32)
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"((uint32_t)BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;
  bool fail = false;

  if (nkb > 0) {
    if (warp == 0 && lane == 0) {
      // producer
      for (int i = 0; i < nkb; ++i) {
        const int s = i % S;
        if (i >= S && !mbar_wait_bounded(&empty[s], (uint32_t)(((i / S) - 1) & 1), kPolls)) {
          fail = true;
          break;
        }
        unsigned char* st = smem + s * STAGE;
        mbar_arrive_expect_tx(&full[s], (uint32_t)STAGE);
        const int kx = (kb0 + i) * KB;
        for (int t = 0; t < T; ++t) tma_load_3d(st + t * A_BYTES, &ta, kx, m0, t, &full[s]);
        for (int t = 0; t < T; ++t) tma_load_3d(st + T * A_BYTES + t * B_BYTES, &tb, kx, n0, t, &full[s]);
      }
    } else if (warp == 1 && lane == 0) {
      // MMA issuer: M=128, N=BN, bf16 x bf16 -> f32, both K-major
      const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
      // three terms: the six leading pairs; two terms: all four pairs (the exact product of
      // the two-term values, so no pair is dropped and the rounding left is unbiased)
      const int ta_[6] = {0, 0, 1, T == 3 ? 0 : 1, 1, 2};
      const int tb_[6] = {0, 1, 0, T == 3 ? 2 : 1, 1, 0};
      for (int i = 0; i < nkb; ++i) {
        const int s = i % S;
        if (!mbar_wait_bounded(&full[s], (uint32_t)((i / S) & 1), kPolls)) {
          fail = true;
          break;
        }
        fence_after();
        unsigned char* st = smem + s * STAGE;
#pragma unroll
        for (int kk = 0; kk < KB / 16; ++kk) {
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            const uint64_t da = swz_desc<KB>(st + ta_[p] * A_BYTES) + (uint64_t)(kk * 2);
            const uint64_t db = swz_desc<KB>(st + T * A_BYTES + tb_[p] * B_BYTES) + (uint64_t)(kk * 2);
            mma_bf16(tmem, da, db, idesc, (i > 0 || kk > 0 || p > 0) ? 1u : 0u);
          }
        }
        mma_commit(&empty[s]);
      }
      mma_commit(done);
    }
  }
  __shared__ int abort_flag;
  if (threadIdx.x == 0) abort_flag = 0;
  __syncthreads();
  if (fail) atomicOr(&abort_flag, 1);
  __syncthreads();
  // epilogue: all four warps
  bool ok = abort_flag == 0;
  if (nkb > 0) ok = mbar_wait_bounded(done, 0u, kPolls) && ok;
  fence_after();
  if (nkb > 0 && ok) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      float v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < o.M) {
        if (o.mode == 0) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            if (col < o.N) {
              const int part = col / o.nsplit;
              double* dst = o.Cp[part] + (long long)row * o.ldc + (col - part * o.nsplit);
              atomicAdd(dst, o.alpha * (double)v[j]);
            }
          }
        } else if (o.mode == 1) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            if (col < o.N) o.Y[(long long)col * o.ldy + row] = v[j];
          }
        } else if (o.mode == 2) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            if (col < o.N) o.Y[(long long)col * o.ldy + row] += v[j];
          }
        } else {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const int col = n0 + c0 + j;  // even: (re, im) of band col / 2
            if (col < o.N)
              *reinterpret_cast<float2*>(o.Y + (long long)(col >> 1) * o.ldy + 2LL * row) = make_float2(v[j], v[j + 1]);
          }
        }
      }
    }
  }
  if (!ok) atomicOr(status, DEV_WAIT_TIMEOUT);
  fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)BN));
}

// ---- operand preparation ----
__device__ __forceinline__ void split3(double x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  a = __double2bfloat16(x);
  const double r = x - (double)__bfloat162float(a);
  b = __double2bfloat16(r);
  c = __double2bfloat16(r - (double)__bfloat162float(b));
}

// planes[t][row][kk] = split(X[row][k0 + kk]) for kk < kc (rows of length ldx); zero pad to kpad.
// sign_swap: complex "B'" operand (x_re, x_im) -> (x_im, -x_re) on the interleaved view.
__global__ void k_split_rows(const float* __restrict__ X, long long ldx, int rows, long long k0, int kc, int kpad,
                             __nv_bfloat16* __restrict__ P, int swap, long long plane, int terms) {
  const long long n = (long long)rows * kpad;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t / kpad), kk = (int)(t % kpad);
    double x = 0.0;
    if (kk < kc) {
      const long long k = k0 + kk;
      if (!swap) {
        x = X[(long long)r * ldx + k];
      } else {
        x = (k & 1) ? -(double)X[(long long)r * ldx + k - 1] : (double)X[(long long)r * ldx + k + 1];
      }
    }
    __nv_bfloat16 a, b, c;
    split3(x, a, b, c);
    P[t] = a;
    P[plane + t] = b;
    if (terms == 3) P[2 * plane + t] = c;
  }
}

// FP32 value into three BF16 terms in FP32 arithmetic: x - bf16(x) and the next remainder are
// exact in FP32, so the terms equal those of the FP64 split of the same value
__device__ __forceinline__ void split3f(float x, __nv_bfloat16& a, __nv_bfloat16& b, __nv_bfloat16& c) {
  a = __float2bfloat16(x);
  const float r = x - __bfloat162float(a);
  b = __float2bfloat16(r);
  c = __float2bfloat16(r - __bfloat162float(b));
}

// k_split_rows for 16-byte aligned rows: four consecutive K values per thread (one 16-byte load,
// one 8-byte store per term plane).  rows * kpad / 4 < 2^31.
__global__ void k_split_rows4(const float* __restrict__ X, long long ldx, int rows, long long k0, int kc, int kpad,
                              __nv_bfloat16* __restrict__ P, long long plane, int terms) {
  const int g4 = kpad >> 2;
  const int n = rows * g4;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int r = t / g4, kk = (t - r * g4) << 2;
    const float* src = X + (long long)r * ldx + k0 + kk;
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    if (kk + 3 < kc) {
      const float4 x = *reinterpret_cast<const float4*>(src);
      v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
      for (int i = 0; i < 4; ++i)
        if (kk + i < kc) v[i] = src[i];
    }
    __align__(8) __nv_bfloat16 a[4], b[4], c[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) split3f(v[i], a[i], b[i], c[i]);
    const long long o = (long long)r * kpad + kk;
    *reinterpret_cast<uint2*>(P + o) = *reinterpret_cast<const uint2*>(a);
    *reinterpret_cast<uint2*>(P + plane + o) = *reinterpret_cast<const uint2*>(b);
    if (terms == 3) *reinterpret_cast<uint2*>(P + 2 * plane + o) = *reinterpret_cast<const uint2*>(c);
  }
}

// planes[t][g][m] = split(X[m][g0 + g]) : transposed chunk (32x32 smem tiles)
__global__ void k_split_transpose(const float* __restrict__ X, long long ldx, int nb, long long g0, int gc, int nbpad,
                                  __nv_bfloat16* __restrict__ P, int terms) {
  __shared__ float tile[32][33];
  const int gx = blockIdx.x * 32, mx = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int m = mx + j, g = gx + threadIdx.x;
    tile[j][threadIdx.x] = (m < nb && g < gc) ? X[(long long)m * ldx + g0 + g] : 0.f;
  }
  __syncthreads();
  const long long plane = (long long)gc * nbpad;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int g = gx + j, m = mx + threadIdx.x;
    if (g < gc && m < nbpad) {
      __nv_bfloat16 a, b, c;
      split3((double)tile[threadIdx.x][j], a, b, c);
      const long long o = (long long)g * nbpad + m;
      P[o] = a;
      P[plane + o] = b;
      if (terms == 3) P[2 * plane + o] = c;
    }
  }
}

// Complex bands (interleaved (re, im) FP32, [nb][ldx] reals): planes[t][g][2 m + c] =
// split(X[m][2 (g0 + g) + c]) for the gc complex points of the chunk, K = 2 nb padded to kpad
// (a 32-band x 16-point tile through shared memory per block).
__global__ void k_split_transpose_c(const float* __restrict__ X, long long ldx, int nb, long long g0, int gc, int kpad,
                                    __nv_bfloat16* __restrict__ P, int terms) {
  __shared__ float tile[32][33];  // [band][real of the 16 points]
  const int gx = blockIdx.x * 16, mx = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int m = mx + j, r = 2 * gx + threadIdx.x;  // real index within the chunk
    tile[j][threadIdx.x] = (m < nb && r < 2 * gc) ? X[(long long)m * ldx + 2 * g0 + r] : 0.f;
  }
  __syncthreads();
  const long long plane = (long long)gc * kpad;
  // output k = 2 (mx + mm) + c for the block's 64 k values, 16 points
  for (int j = threadIdx.y; j < 16; j += blockDim.y) {
    const int g = gx + j;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int kk = threadIdx.x + 32 * h;  // 0..63 within the block
      const int mm = kk >> 1, c = kk & 1;
      const int k = 2 * mx + kk;
      if (g < gc && k < kpad) {
        __nv_bfloat16 a, b, cc;
        split3((double)tile[mm][2 * j + c], a, b, cc);
        const long long o = (long long)g * kpad + k;
        P[o] = a;
        P[plane + o] = b;
        if (terms == 3) P[2 * plane + o] = cc;
      }
    }
  }
}

// W (2 nb x 2 nb, column-major, FP64): the real form of the complex rotation C (nb x nb,
// column-major interleaved) acting on (re, im) pairs: new_re_j = sum_m re_m Cr_mj - im_m Ci_mj,
// new_im_j = sum_m re_m Ci_mj + im_m Cr_mj, with input k = 2 m + c and output n = 2 j + c'.
__global__ void k_complex_rotation_real(const double* __restrict__ Cz, int nb, double* __restrict__ W) {
  const long long n2 = 2LL * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n2 * n2; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % n2), n = (int)(t / n2);
    const int m = k >> 1, c = k & 1, j = n >> 1, cp = n & 1;
    const double cr = Cz[2 * ((long long)m + (long long)j * nb)], ci = Cz[2 * ((long long)m + (long long)j * nb) + 1];
    W[t] = cp == 0 ? (c == 0 ? cr : -ci) : (c == 0 ? ci : cr);
  }
}

// planes[t][n][m] = split(V[m + n*ldv]) (V column-major FP64 = row-major V^T)
__global__ void k_split_small(const double* __restrict__ V, int ldv, int nb, int nbpad, __nv_bfloat16* __restrict__ P,
                              int terms) {
  const long long plane = (long long)nb * nbpad;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < plane; t += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(t / nbpad), m = (int)(t % nbpad);
    const double x = m < nb ? V[m + (long long)n * ldv] : 0.0;
    __nv_bfloat16 a, b, c;
    split3(x, a, b, c);
    P[t] = a;
    P[plane + t] = b;
    if (terms == 3) P[2 * plane + t] = c;
  }
}

}  // namespace x3

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static int get_encode() {
  if (g_encode) return 0;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  RS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  RS_CHECK(fn != nullptr && q == cudaDriverEntryPointSuccess, RSDFT_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return 0;
}

// Tile shape of a contraction: three terms, 128 x 128 tiles in K blocks of 64 (2 stages of
// 96 KB) or, wide (the default), 128 x 256 tiles in K blocks of 32 (3 stages of 72 KB: each
// operand byte feeds twice the products); two terms, 128 x 256 tiles in K blocks of 64.
struct TileCfg {
  int bn, kb;
};
static TileCfg tile_for(const Ctx& c, int terms) {
  if (terms == 2) return {256, 64};
  return c.gemm_wide ? TileCfg{256, 32} : TileCfg{128, 64};
}

// 3-D map over [planes][rows][kpad] bf16 (plane stride plane_rows x kpad), box {kb, box_rows, 1},
// 128B swizzle (kb = 64) or 64B swizzle (kb = 32)
static int make_map(CUtensorMap* m, const void* base, long long rows, long long kpad, int box_rows, int planes,
                    long long plane_rows, int kb) {
  RS_TRY(get_encode());
  cuuint64_t dims[3] = {(cuuint64_t)kpad, (cuuint64_t)rows, (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)kpad * 2, (cuuint64_t)plane_rows * kpad * 2};
  cuuint32_t box[3] = {(cuuint32_t)kb, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        kb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  RS_CHECK(r == CUDA_SUCCESS, RSDFT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return 0;
}

template <int BN, int S, int T, int KB>
static int launch_x3(Ctx& c, const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, long long kpad,
                     const x3::Out& o, int ksplit) {
  const int kbt = (int)(kpad / KB);
  const int kps = (kbt + ksplit - 1) / ksplit;
  ksplit = (kbt + kps - 1) / kps;
  constexpr int STAGE = T * x3::BM * KB * 2 + T * BN * KB * 2;
  const size_t smem = (size_t)S * STAGE + 1024 + 256;
  auto kern = x3::k_gemm_x3<BN, S, T, KB>;
  static bool attr = false;
  if (!attr) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  dim3 grid((M + x3::BM - 1) / x3::BM, (N + BN - 1) / BN, ksplit);
  kern<<<grid, x3::kThreads, smem, c.stream>>>(ta, tb, kbt, kps, o, c.d_status);
  c.launches++;
  return check_launch("gemm_x3");
}

static int launch_terms(Ctx& c, int terms, const CUtensorMap& ta, const CUtensorMap& tb, int M, int N, long long kpad,
                        const x3::Out& o, int ksplit) {
  const TileCfg t = tile_for(c, terms);
  if (terms == 2) return launch_x3<256, 2, 2, 64>(c, ta, tb, M, N, kpad, o, ksplit);
  if (t.bn == 256) return launch_x3<256, 3, 3, 32>(c, ta, tb, M, N, kpad, o, ksplit);
  return launch_x3<128, 2, 3, 64>(c, ta, tb, M, N, kpad, o, ksplit);
}

// X rows [0, rows) from column k0 into the term planes (pstride elements apart) of one chunk
static void split_rows(Ctx& c, const float* X, long long ldx, int rows, long long k0, int kc, int kpad,
                       __nv_bfloat16* P, int swap, long long pstride, int terms) {
  const bool vec = !swap && (reinterpret_cast<uintptr_t>(X) & 15) == 0 && ldx % 4 == 0 && k0 % 4 == 0 &&
                   (long long)rows * (kpad / 4) < (1LL << 31);
  if (vec)
    x3::k_split_rows4<<<8 * 148, 256, 0, c.stream>>>(X, ldx, rows, k0, kc, kpad, P, pstride, terms);
  else
    x3::k_split_rows<<<4 * 148, 256, 0, c.stream>>>(X, ldx, rows, k0, kc, kpad, P, swap, pstride, terms);
  c.launches++;
}

// Split-K chunk of a contraction with rows_total operand rows: the BF16 planes of one chunk stay
// within 512 MB.
static long long chunk_k(long long rows_total, int terms, long long K) {
  const long long kc_max = std::max<long long>(64, ((long long)(512u << 20) / (2LL * terms * rows_total)) / 64 * 64);
  return std::min<long long>(kc_max, (K + 63) / 64 * 64);
}

static int split_ksplit(int M, int N, int kpad, int bn, bool tri = false) {
  int tiles = ((M + 127) / 128) * ((N + bn - 1) / bn);
  if (tri) tiles = std::max(1, tiles * 3 / 4);  // about a quarter of the tiles (half of S) are left out
  const int kbt = kpad / 64;
  return std::max(1, std::min(kbt, (2 * 148 + tiles - 1) / tiles));
}

// C[m][n] += alpha * sum_k A[m][k] B[n][k]; A: [M][lda] FP32, B: [N][ldb] FP32 (real view).
// swapB: B is read as the complex "i-rotated" view (b_re, b_im) -> (b_im, -b_re).
// terms: 3 (about FP32 accuracy) or 2 (see the head of this file).
int gemm_tn_x3(Ctx& c, const float* A, long long lda, int M, const float* B, long long ldb, int N, long long K,
               double alpha, double* C, long long ldc, int swapB, int terms) {
  RS_CHECK(terms == 2 || terms == 3, RSDFT_ERR_ARG, "split terms must be 2 or 3");
  const long long kc = chunk_k(M + N, terms, K);
  RS_TRY(c.ws_gemm.ensure(sizeof(__nv_bfloat16) * terms * (size_t)(M + N) * kc));
  __nv_bfloat16* PA = c.ws_gemm.as<__nv_bfloat16>();
  __nv_bfloat16* PB = PA + terms * (size_t)M * kc;
  const double flops = 2.0 * (terms == 3 ? 6.0 : 4.0) * (double)M * N * K;
  ProfScope ps(c, "gemm", 0.0, flops);
  for (long long k0 = 0; k0 < K; k0 += kc) {
    const int kcur = (int)std::min<long long>(kc, K - k0);
    const int kpad = (kcur + 63) / 64 * 64;
    split_rows(c, A, lda, M, k0, kcur, kpad, PA, 0, (long long)M * kpad, terms);
    split_rows(c, B, ldb, N, k0, kcur, kpad, PB, swapB, (long long)N * kpad, terms);
    RS_TRY(check_launch("split_rows"));
    CUtensorMap ta, tb;
    const TileCfg tc = tile_for(c, terms);
    RS_TRY(make_map(&ta, PA, M, kpad, x3::BM, terms, M, tc.kb));
    RS_TRY(make_map(&tb, PB, N, kpad, tc.bn, terms, N, tc.kb));
    x3::Out o{};
    o.mode = 0; o.Cp[0] = C; o.nsplit = N; o.ldc = ldc; o.alpha = alpha; o.M = M; o.N = N;
    RS_TRY(launch_terms(c, terms, ta, tb, M, N, kpad, o, split_ksplit(M, N, kpad, tc.bn)));
  }
  return 0;
}

// S[m][n] += alpha * sum_k X[m][k] X[n][k] and M[m][n] += alpha * sum_k X[m][k] Y[n][k] in one
// contraction of X against [X; Y] (N = 2 nb): X is split once per chunk and serves as A and as
// the first nb rows of B.  X, Y: [nb][ld] FP32; S, M: nb x nb, leading dimension nb.  Both are
// symmetric (Y = H X with H symmetric), so only the tiles reaching n <= m are formed: complete
// for n <= m (the upper triangle of the column-major matrices), partial above.
int gemm_tn2_x3(Ctx& c, const float* X, const float* Y, long long ld, int nb, long long K, double alpha, double* S,
                double* M, int terms) {
  RS_CHECK(terms == 2 || terms == 3, RSDFT_ERR_ARG, "split terms must be 2 or 3");
  const long long kc = chunk_k(2LL * nb, terms, K);
  RS_TRY(c.ws_gemm.ensure(sizeof(__nv_bfloat16) * terms * (size_t)(2 * nb) * kc));
  __nv_bfloat16* P = c.ws_gemm.as<__nv_bfloat16>();
  const double flops = 2.0 * (terms == 3 ? 6.0 : 4.0) * (double)nb * (2.0 * nb) * K;
  ProfScope ps(c, "gemm", 0.0, flops);
  for (long long k0 = 0; k0 < K; k0 += kc) {
    const int kcur = (int)std::min<long long>(kc, K - k0);
    const int kpad = (kcur + 63) / 64 * 64;
    const long long plane = 2LL * nb * kpad;  // [terms][2 nb][kpad]: rows of X, then rows of Y
    split_rows(c, X, ld, nb, k0, kcur, kpad, P, 0, plane, terms);
    split_rows(c, Y, ld, nb, k0, kcur, kpad, P + (size_t)nb * kpad, 0, plane, terms);
    RS_TRY(check_launch("split_rows"));
    CUtensorMap ta, tb;
    const TileCfg tc = tile_for(c, terms);
    RS_TRY(make_map(&ta, P, nb, kpad, x3::BM, terms, 2LL * nb, tc.kb));
    RS_TRY(make_map(&tb, P, 2LL * nb, kpad, tc.bn, terms, 2LL * nb, tc.kb));
    x3::Out o{};
    o.mode = 0; o.Cp[0] = S; o.Cp[1] = M; o.nsplit = nb; o.ldc = nb; o.alpha = alpha; o.M = nb; o.N = 2 * nb;
    o.tri = c.gemm_tri;  // 0, 1 (S by triangle tiles) or 2 (S and Hsub)
    RS_TRY(launch_terms(c, terms, ta, tb, nb, 2 * nb, kpad, o, split_ksplit(nb, 2 * nb, kpad, tc.bn, c.gemm_tri != 0)));
  }
  return 0;
}

// X[n][g] <- sum_m X[m][g] V[m][n] for all g (in place, grid chunks); X: [nb][ldx] FP32,
// V: nb x nb FP64 column-major (ldv).  add: X[n][g] <- X[n][g] + sum_m X[m][g] V[m][n] (the
// update form X (I + V): with V small the FP32 accumulation error scales with |X V|, not |X|).
int gemm_rotate_x3(Ctx& c, float* X, long long ldx, int nb, long long G, const double* V, int ldv, int terms,
                   bool add) {
  RS_CHECK(terms == 2 || terms == 3, RSDFT_ERR_ARG, "split terms must be 2 or 3");
  const int nbpad = (nb + 63) / 64 * 64;
  const long long gc_max = std::max<long long>(128, ((long long)(512u << 20) / (2LL * terms * nbpad)) / 128 * 128);
  const long long gc = std::min<long long>(gc_max, (G + 127) / 128 * 128);
  RS_TRY(c.ws_gemm.ensure(sizeof(__nv_bfloat16) * terms * ((size_t)gc * nbpad + (size_t)nb * nbpad)));
  __nv_bfloat16* PV = c.ws_gemm.as<__nv_bfloat16>();
  __nv_bfloat16* PX = PV + terms * (size_t)nb * nbpad;
  const double flops = 2.0 * (terms == 3 ? 6.0 : 4.0) * (double)nb * nb * G;
  ProfScope ps(c, "gemm", 0.0, flops);
  x3::k_split_small<<<4 * 148, 256, 0, c.stream>>>(V, ldv, nb, nbpad, PV, terms);
  c.launches++;
  CUtensorMap tb;
  const TileCfg tc = tile_for(c, terms);
  RS_TRY(make_map(&tb, PV, nb, nbpad, tc.bn, terms, nb, tc.kb));
  for (long long g0 = 0; g0 < G; g0 += gc) {
    const int gcur = (int)std::min<long long>(gc, G - g0);
    dim3 tg((gcur + 31) / 32, (nbpad + 31) / 32);
    x3::k_split_transpose<<<tg, dim3(32, 8), 0, c.stream>>>(X, ldx, nb, g0, gcur, nbpad, PX, terms);
    c.launches++;
    RS_TRY(check_launch("split_transpose"));
    CUtensorMap ta;
    RS_TRY(make_map(&ta, PX, gcur, nbpad, x3::BM, terms, gcur, tc.kb));
    x3::Out o{};
    o.mode = add ? 2 : 1; o.Y = X + g0; o.ldy = ldx; o.M = gcur; o.N = nb;
    RS_TRY(launch_terms(c, terms, ta, tb, gcur, nb, nbpad, o, 1));
  }
  return 0;
}

// Cp[p][m][n] += alpha * sum_k A[m][k] B_p[n][k] for the parts p < nparts of B (np rows each,
// read as is or, swap[p], as the complex i-rotated view), in one contraction of A against the
// stacked parts: A is split once per K chunk.  A: [M][lda], B_p: [np][ldb] FP32 real views;
// Cp[p]: M x np row-major (ldc).
int gemm_tn_cat_x3(Ctx& c, const float* A, long long lda, int M, const float* const* B, const int* swap, int nparts,
                   long long ldb, int np, long long K, double alpha, double* const* Cp, long long ldc, int terms) {
  RS_CHECK(terms == 2 || terms == 3, RSDFT_ERR_ARG, "split terms must be 2 or 3");
  RS_CHECK(nparts >= 1 && nparts <= 4, RSDFT_ERR_ARG, "1 to 4 operand parts");
  const int N = nparts * np;
  const long long kc = chunk_k(M + N, terms, K);
  RS_TRY(c.ws_gemm.ensure(sizeof(__nv_bfloat16) * terms * (size_t)(M + N) * kc));
  __nv_bfloat16* PA = c.ws_gemm.as<__nv_bfloat16>();
  __nv_bfloat16* PB = PA + terms * (size_t)M * kc;
  const double flops = 2.0 * (terms == 3 ? 6.0 : 4.0) * (double)M * N * K;
  ProfScope ps(c, "gemm", 0.0, flops);
  for (long long k0 = 0; k0 < K; k0 += kc) {
    const int kcur = (int)std::min<long long>(kc, K - k0);
    const int kpad = (kcur + 63) / 64 * 64;
    split_rows(c, A, lda, M, k0, kcur, kpad, PA, 0, (long long)M * kpad, terms);
    for (int p = 0; p < nparts; ++p)
      split_rows(c, B[p], ldb, np, k0, kcur, kpad, PB + (size_t)p * np * kpad, swap[p], (long long)N * kpad, terms);
    RS_TRY(check_launch("split_rows"));
    CUtensorMap ta, tb;
    const TileCfg tc = tile_for(c, terms);
    RS_TRY(make_map(&ta, PA, M, kpad, x3::BM, terms, M, tc.kb));
    RS_TRY(make_map(&tb, PB, N, kpad, tc.bn, terms, N, tc.kb));
    x3::Out o{};
    o.mode = 0;
    for (int p = 0; p < nparts; ++p) o.Cp[p] = Cp[p];
    o.nsplit = np; o.ldc = ldc; o.alpha = alpha; o.M = M; o.N = N;
    RS_TRY(launch_terms(c, terms, ta, tb, M, N, kpad, o, split_ksplit(M, N, kpad, tc.bn)));
  }
  return 0;
}

// Complex bands X (nb bands of G complex points, interleaved FP32, leading dimension ldx reals)
// rotated in place: X[j](g) <- sum_m X[m](g) C[m][j], C nb x nb complex column-major (ldc = nb),
// as a real contraction over K = 2 nb: the (re, im) pairs of the nb input bands against the real
// 2 nb x 2 nb form of C.
int gemm_rotate_cx3(Ctx& c, float* X, long long ldx, int nb, long long G, const double* Cz, int terms) {
  RS_CHECK(terms == 2 || terms == 3, RSDFT_ERR_ARG, "split terms must be 2 or 3");
  const int n2 = 2 * nb;
  const int kpad = (n2 + 63) / 64 * 64;
  const long long gc_max = std::max<long long>(128, ((long long)(512u << 20) / (2LL * terms * kpad)) / 128 * 128);
  const long long gc = std::min<long long>(gc_max, (G + 127) / 128 * 128);
  RS_TRY(c.ws_gemm.ensure(sizeof(__nv_bfloat16) * terms * ((size_t)gc * kpad + (size_t)n2 * kpad)));
  RS_TRY(c.ws_rot.ensure(sizeof(double) * (size_t)n2 * n2));
  __nv_bfloat16* PV = c.ws_gemm.as<__nv_bfloat16>();
  __nv_bfloat16* PX = PV + terms * (size_t)n2 * kpad;
  const double flops = 2.0 * (terms == 3 ? 6.0 : 4.0) * (double)n2 * n2 * G;
  ProfScope ps(c, "gemm", 0.0, flops);
  double* Wr = c.ws_rot.as<double>();
  x3::k_complex_rotation_real<<<4 * 148, 256, 0, c.stream>>>(Cz, nb, Wr);
  x3::k_split_small<<<4 * 148, 256, 0, c.stream>>>(Wr, n2, n2, kpad, PV, terms);
  c.launches += 2;
  CUtensorMap tb;
  const TileCfg tc = tile_for(c, terms);
  RS_TRY(make_map(&tb, PV, n2, kpad, tc.bn, terms, n2, tc.kb));
  for (long long g0 = 0; g0 < G; g0 += gc) {
    const int gcur = (int)std::min<long long>(gc, G - g0);
    dim3 tg((gcur + 15) / 16, (kpad / 2 + 31) / 32);
    x3::k_split_transpose_c<<<tg, dim3(32, 8), 0, c.stream>>>(X, ldx, nb, g0, gcur, kpad, PX, terms);
    c.launches++;
    RS_TRY(check_launch("split_transpose_c"));
    CUtensorMap ta;
    RS_TRY(make_map(&ta, PX, gcur, kpad, x3::BM, terms, gcur, tc.kb));
    x3::Out o{};
    o.mode = 3; o.Y = X + 2 * g0; o.ldy = ldx; o.M = gcur; o.N = n2;
    RS_TRY(launch_terms(c, terms, ta, tb, gcur, n2, kpad, o, 1));
  }
  return 0;
}

}  // namespace rsdft

// ---------------------------------------------------------------------------
// self-test against cuBLAS DGEMM on the same FP32 inputs (diagnostic entry)
// ---------------------------------------------------------------------------
namespace rsdft {
namespace x3 {
__global__ void k_fill(float* a, long long n, unsigned long long seed) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(t + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    a[t] = (float)((double)(z >> 11) * 0x1.0p-53 - 0.5);
  }
}
__global__ void k_f2d_x3(const float* s, double* d, long long n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    d[t] = (double)s[t];
}
}  // namespace x3

int selftest_gemm(Ctx& c, int m, int n, long long k, int op, int terms, double* err) {
  DBuf a, b, ad, bd, cc, cref, v;
  const long long na = op == 0 ? (long long)m * k : (long long)m * k;  // op1: X [m=nb][k=G]
  const long long nbv = op == 0 ? (long long)n * k : op == 2 ? (long long)m * k : (long long)m * m;
  RS_TRY(a.ensure(sizeof(float) * na));
  RS_TRY(ad.ensure(sizeof(double) * na));
  RS_TRY(b.ensure(sizeof(float) * nbv));
  RS_TRY(bd.ensure(sizeof(double) * nbv));
  x3::k_fill<<<256, 256, 0, c.stream>>>(a.as<float>(), na, 11);
  x3::k_fill<<<256, 256, 0, c.stream>>>(b.as<float>(), nbv, 23);
  x3::k_f2d_x3<<<256, 256, 0, c.stream>>>(a.as<float>(), ad.as<double>(), na);
  x3::k_f2d_x3<<<256, 256, 0, c.stream>>>(b.as<float>(), bd.as<double>(), nbv);
  const double one = 1.0, zero = 0.0;
  std::vector<double> h1, h2;
  if (op == 2) {
    // fused [S | M] = [A A^T | A B^T] (B: m x k) through gemm_tn2_x3, against DGEMM on the
    // elements the contraction guarantees (n <= m when only triangle tiles are formed)
    RS_CHECK(n == m, RSDFT_ERR_ARG, "op 2 needs n == m");
    RS_TRY(cc.ensure(sizeof(double) * 2 * (size_t)m * m));
    RS_TRY(cref.ensure(sizeof(double) * 2 * (size_t)m * m));
    RS_CUDA(cudaMemsetAsync(cc.p, 0, sizeof(double) * 2 * (size_t)m * m, c.stream));
    RS_TRY(gemm_tn2_x3(c, a.as<float>(), b.as<float>(), k, m, k, 1.0, cc.as<double>(),
                       cc.as<double>() + (size_t)m * m, terms));
    double* rS = cref.as<double>();
    double* rM = rS + (size_t)m * m;
    if (cublasDgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, (int)k, &one, ad.as<double>(), (int)k, ad.as<double>(),
                    (int)k, &zero, rS, m) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, (int)k, &one, ad.as<double>(), (int)k, bd.as<double>(),
                    (int)k, &zero, rM, m) != CUBLAS_STATUS_SUCCESS)
      RS_CHECK(false, RSDFT_ERR_CUDA, "reference dgemm failed");
    h1.resize(2 * (size_t)m * m);
    h2.resize(2 * (size_t)m * m);
    RS_CUDA(cudaMemcpyAsync(h1.data(), cc.p, sizeof(double) * h1.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaMemcpyAsync(h2.data(), cref.p, sizeof(double) * h2.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    double mx = 0.0, me = 0.0;
    for (int part = 0; part < 2; ++part)
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          if (j > i && (c.gemm_tri == 2 || (c.gemm_tri == 1 && part == 0))) continue;
          const double r = h2[(size_t)part * m * m + i + (size_t)j * m];
          mx = std::max(mx, std::fabs(r));
          me = std::max(me, std::fabs(h1[(size_t)part * m * m + (size_t)i * m + j] - r));
        }
    *err = me / std::max(mx, 1e-300);
  } else if (op == 0) {
    RS_TRY(cc.ensure(sizeof(double) * (size_t)m * n));
    RS_TRY(cref.ensure(sizeof(double) * (size_t)m * n));
    RS_CUDA(cudaMemsetAsync(cc.p, 0, sizeof(double) * (size_t)m * n, c.stream));
    RS_TRY(gemm_tn_x3(c, a.as<float>(), k, m, b.as<float>(), k, n, k, 1.0, cc.as<double>(), n, 0, terms));
    // reference, column-major m x n: C_cm = A_cm^T B_cm with A_cm (k x m), B_cm (k x n)
    if (cublasDgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, n, (int)k, &one, ad.as<double>(), (int)k, bd.as<double>(),
                    (int)k, &zero, cref.as<double>(), m) != CUBLAS_STATUS_SUCCESS)
      RS_CHECK(false, RSDFT_ERR_CUDA, "reference dgemm failed");
    h1.resize((size_t)m * n);
    h2.resize((size_t)m * n);
    RS_CUDA(cudaMemcpyAsync(h1.data(), cc.p, sizeof(double) * h1.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaMemcpyAsync(h2.data(), cref.p, sizeof(double) * h2.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    double mx = 0.0, me = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < n; ++j) {
        const double r = h2[i + (size_t)j * m];
        mx = std::max(mx, std::fabs(r));
        me = std::max(me, std::fabs(h1[(size_t)i * n + j] - r));
      }
    *err = me / std::max(mx, 1e-300);
  } else {
    // X [m][k] rotated by V (m x m, column-major); reference Y_cm = X_cm V
    RS_TRY(cref.ensure(sizeof(double) * (size_t)na));
    RS_TRY(v.ensure(sizeof(double) * (size_t)m * m));
    RS_CUDA(cudaMemcpyAsync(v.p, bd.p, sizeof(double) * (size_t)m * m, cudaMemcpyDeviceToDevice, c.stream));
    if (cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)k, m, m, &one, ad.as<double>(), (int)k, v.as<double>(), m,
                    &zero, cref.as<double>(), (int)k) != CUBLAS_STATUS_SUCCESS)
      RS_CHECK(false, RSDFT_ERR_CUDA, "reference dgemm failed");
    RS_TRY(gemm_rotate_x3(c, a.as<float>(), k, m, k, v.as<double>(), m, terms, false));
    std::vector<float> hy((size_t)na);
    h2.resize((size_t)na);
    RS_CUDA(cudaMemcpyAsync(hy.data(), a.p, sizeof(float) * hy.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaMemcpyAsync(h2.data(), cref.p, sizeof(double) * h2.size(), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    double mx = 0.0, me = 0.0;
    for (size_t t = 0; t < (size_t)na; ++t) {
      mx = std::max(mx, std::fabs(h2[t]));
      me = std::max(me, std::fabs((double)hy[t] - h2[t]));
    }
    *err = me / std::max(mx, 1e-300);
  }
  a.release(); b.release(); ad.release(); bd.release(); cc.release(); cref.release(); v.release();
  return check_launch("selftest_gemm");
}
}  // namespace rsdft
