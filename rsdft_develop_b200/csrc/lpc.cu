// Learned preconditioner: a 4-layer 3-D convolutional network that maps a band gradient g to
// a search direction, standing in for precond_hprsdft
// (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270) in the CG band update.
//
// Network: channels 1 -> 16 -> 16 -> 16 -> 1, 3x3x3 kernels, no biases, tanh after the first
// three layers.  Without biases and with an odd activation the map is odd, f(-g) = -f(g), and
// the input is scaled by its RMS before and the output by the same factor after, so the
// preconditioner is sign- and scale-equivariant like the plain one.  Weights are kept in
// FP32 (Adam master copy) and used as BF16; all convolutions accumulate in FP32.
//
// Kernels (all hand-written here):
//   k_conv_fwd<CIN,COUT,ACT,DACT>  'same' 3x3x3 convolution (periodic or zero padding) of a
//       [batch][C][n3][n2][n1] tensor on 16x8x2 output tiles staged with a one-point halo in
//       shared memory; optional tanh epilogue (forward) or (1 - a^2) epilogue (backward).
//   backward-data = k_conv_fwd with transposed, flipped weights (adjoint of a 'same' conv).
//   k_conv_bwd_w<CIN,COUT>  dW[co][ci][tap] = sum dz[co](p) x[ci](p + tap), one (co,ci) pair
//       per thread accumulated over many tiles, then added into FP32 gradients.
//   k_loss  MSE on the patch interior (a margin of the receptive-field radius), dL/dy.
//   k_adam  Adam update of the FP32 master weights and their BF16 copy.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <random>

#include "ctx.cuh"
#include "ptx.cuh"

namespace rsdft {
namespace lpc {

constexpr int NL = 4;
constexpr int CH[NL + 1] = {1, 16, 16, 16, 1};
constexpr int TX = 16, TY = 8, TZ = 2;  // output tile: 256 points, one per thread
constexpr int NTHR = TX * TY * TZ;
constexpr int WTOT = 27 * (16 * 1 + 16 * 16 + 16 * 16 + 1 * 16);  // 14688
static_assert(WTOT == RSDFT_LPC_NWEIGHTS, "weight count differs from the C header");

constexpr int woff(int l) {
  int o = 0;
  for (int j = 0; j < l; ++j) o += 27 * CH[j] * CH[j + 1];
  return o;
}

struct Dims {
  int n1, n2, n3;
  int periodic;
  int tiles_x, tiles_y, tiles_z;
};

__device__ __forceinline__ int wrap(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HVOL = HX * HY * HZ;
constexpr int CS = HVOL + 1;  // per-channel stride of a staged tile (odd: channels land in distinct banks)

template <int CIN>
__device__ __forceinline__ void load_tile(float* xs, const float* __restrict__ in, const Dims& d, int x0, int y0, int z0) {
  const size_t plane = (size_t)d.n1 * d.n2, vol = plane * d.n3;
  for (int e = threadIdx.x; e < CIN * HVOL; e += NTHR) {
    const int hx = e % HX, hy = (e / HX) % HY, hz = (e / (HX * HY)) % HZ, c = e / HVOL;
    int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
    float v = 0.f;
    if (d.periodic) {
      gx = wrap(gx, d.n1); gy = wrap(gy, d.n2); gz = wrap(gz, d.n3);
      v = __ldg(in + c * vol + gz * plane + (size_t)gy * d.n1 + gx);
    } else if (gx >= 0 && gx < d.n1 && gy >= 0 && gy < d.n2 && gz >= 0 && gz < d.n3) {
      v = __ldg(in + c * vol + gz * plane + (size_t)gy * d.n1 + gx);
    }
    xs[c * CS + (e - c * HVOL)] = v;
  }
}

// out = act(conv(in, w)); DACT: out = conv(in, w) * (1 - a^2) with a the given activations
template <int CIN, int COUT, bool ACT, bool DACT>
__global__ void __launch_bounds__(NTHR) k_conv_fwd(const float* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                   float* __restrict__ out, const float* __restrict__ act_in, Dims d) {
  extern __shared__ float sm[];
  float* ws = sm;                       // [COUT][CIN][27]
  float* xs = sm + COUT * CIN * 27;     // [CIN][CS] halo tiles
  for (int e = threadIdx.x; e < COUT * CIN * 27; e += NTHR) ws[e] = __bfloat162float(w[e]);
  const int t = blockIdx.x;
  const int bx = t % d.tiles_x, by = (t / d.tiles_x) % d.tiles_y, bz = t / (d.tiles_x * d.tiles_y);
  const int x0 = bx * TX, y0 = by * TY, z0 = bz * TZ;
  const size_t plane = (size_t)d.n1 * d.n2, vol = plane * d.n3;
  const float* inb = in + (size_t)blockIdx.y * CIN * vol;
  load_tile<CIN>(xs, inb, d, x0, y0, z0);
  __syncthreads();
  const int tx = threadIdx.x % TX, ty = (threadIdx.x / TX) % TY, tz = threadIdx.x / (TX * TY);
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = 0.f;
  for (int ci = 0; ci < CIN; ++ci) {
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const float v = xs[ci * CS + ((tz + kz) * HY + ty + ky) * HX + tx + kx];
          const int tap = (kz * 3 + ky) * 3 + kx;
#pragma unroll
          for (int co = 0; co < COUT; ++co) acc[co] += ws[(co * CIN + ci) * 27 + tap] * v;
        }
  }
  const int gx = x0 + tx, gy = y0 + ty, gz = z0 + tz;
  if (gx < d.n1 && gy < d.n2 && gz < d.n3) {
    const size_t o = (size_t)gz * plane + (size_t)gy * d.n1 + gx;
    float* ob = out + (size_t)blockIdx.y * COUT * vol;
#pragma unroll
    for (int co = 0; co < COUT; ++co) {
      float r = acc[co];
      if (ACT) r = tanhf(r);
      if (DACT) {
        const float a = act_in[(size_t)blockIdx.y * COUT * vol + co * vol + o];
        r *= (1.f - a * a);
      }
      ob[co * vol + o] = r;
    }
  }
}

// Faster 'same' convolution for COUT a multiple of 2 (same contract as k_conv_fwd): output tile
// 16 x 8 x 8, each thread 4 consecutive z outputs x COUT channels accumulated as float2 pairs
// of channels with packed FMAs; input channels staged 8 at a time; weights as [ci][tap][co].
constexpr int FX = 16, FY = 8, FZ = 8, FCC = 8;
constexpr int FHX = FX + 2, FHY = FY + 2, FHZ = FZ + 2;
constexpr int FCS = FHX * FHY * FHZ + 4;  // per-channel stride (keeps float4 alignment)

template <int CIN, int COUT, bool ACT, bool DACT>
__global__ void __launch_bounds__(256, 1) k_conv_fwd4(const float* __restrict__ in, const __nv_bfloat16* __restrict__ w,
                                                   float* __restrict__ out, const float* __restrict__ act_in, Dims d,
                                                   int tiles_x, int tiles_y) {
  static_assert(COUT % 2 == 0, "pairs of output channels");
  constexpr int CC = CIN < FCC ? CIN : FCC;
  extern __shared__ __align__(16) float sm[];
  float* ws = sm;                 // [CC][27][COUT]
  float* xs = sm + CC * 27 * COUT;  // [CC][FCS]
  const int t = blockIdx.x;
  const int bx = t % tiles_x, by = (t / tiles_x) % tiles_y, bz = t / (tiles_x * tiles_y);
  const int x0 = bx * FX, y0 = by * FY, z0 = bz * FZ;
  const size_t plane = (size_t)d.n1 * d.n2, vol = plane * d.n3;
  const float* inb = in + (size_t)blockIdx.y * CIN * vol;
  const int tx = threadIdx.x % FX, ty = (threadIdx.x / FX) % FY, tq = threadIdx.x / (FX * FY);  // tq: z quarter 0..1
  float2 acc[4][COUT / 2];
#pragma unroll
  for (int zi = 0; zi < 4; ++zi)
#pragma unroll
    for (int c = 0; c < COUT / 2; ++c) acc[zi][c] = make_float2(0.f, 0.f);
  for (int c0 = 0; c0 < CIN; c0 += CC) {
    __syncthreads();
    for (int e = threadIdx.x; e < CC * 27 * COUT; e += 256) {
      const int co = e % COUT, tap = (e / COUT) % 27, ci = e / (27 * COUT);
      ws[e] = __bfloat162float(w[(co * CIN + c0 + ci) * 27 + tap]);
    }
    for (int e = threadIdx.x; e < CC * FHX * FHY * FHZ; e += 256) {
      const int hx = e % FHX, hy = (e / FHX) % FHY, hz = (e / (FHX * FHY)) % FHZ, c = e / (FHX * FHY * FHZ);
      int gx = x0 - 1 + hx, gy = y0 - 1 + hy, gz = z0 - 1 + hz;
      float v = 0.f;
      if (d.periodic) {
        gx = wrap(gx, d.n1); gy = wrap(gy, d.n2); gz = wrap(gz, d.n3);
        v = __ldg(inb + (size_t)(c0 + c) * vol + gz * plane + (size_t)gy * d.n1 + gx);
      } else if (gx >= 0 && gx < d.n1 && gy >= 0 && gy < d.n2 && gz >= 0 && gz < d.n3) {
        v = __ldg(inb + (size_t)(c0 + c) * vol + gz * plane + (size_t)gy * d.n1 + gx);
      }
      xs[c * FCS + (e - c * FHX * FHY * FHZ)] = v;
    }
    __syncthreads();
    for (int ci = 0; ci < CC; ++ci) {
      const float* xc = xs + ci * FCS;
#pragma unroll
      for (int ky = 0; ky < 3; ++ky)
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          float xv[6];
#pragma unroll
          for (int j = 0; j < 6; ++j) xv[j] = xc[((tq * 4 + j) * FHY + ty + ky) * FHX + tx + kx];
#pragma unroll
          for (int kz = 0; kz < 3; ++kz) {
            const float* wt = ws + (ci * 27 + (kz * 3 + ky) * 3 + kx) * COUT;
#pragma unroll
            for (int c4 = 0; c4 < COUT / 4; ++c4) {
              const float4 w4 = *reinterpret_cast<const float4*>(wt + 4 * c4);
              const float2 wa = make_float2(w4.x, w4.y), wb = make_float2(w4.z, w4.w);
#pragma unroll
              for (int zi = 0; zi < 4; ++zi) {
                const float2 xx = make_float2(xv[zi + kz], xv[zi + kz]);
                acc[zi][2 * c4] = __ffma2_rn(wa, xx, acc[zi][2 * c4]);
                acc[zi][2 * c4 + 1] = __ffma2_rn(wb, xx, acc[zi][2 * c4 + 1]);
              }
            }
            if constexpr (COUT % 4 == 2) {
              const float2 wa = *reinterpret_cast<const float2*>(wt + COUT - 2);
#pragma unroll
              for (int zi = 0; zi < 4; ++zi)
                acc[zi][COUT / 2 - 1] = __ffma2_rn(wa, make_float2(xv[zi + kz], xv[zi + kz]), acc[zi][COUT / 2 - 1]);
            }
          }
        }
    }
  }
  const int gx = x0 + tx, gy = y0 + ty;
  if (gx >= d.n1 || gy >= d.n2) return;
  float* ob = out + (size_t)blockIdx.y * COUT * vol;
#pragma unroll
  for (int zi = 0; zi < 4; ++zi) {
    const int gz = z0 + tq * 4 + zi;
    if (gz >= d.n3) break;
    const size_t o = (size_t)gz * plane + (size_t)gy * d.n1 + gx;
#pragma unroll
    for (int c = 0; c < COUT; ++c) {
      float r = (c & 1) ? acc[zi][c / 2].y : acc[zi][c / 2].x;
      if (ACT) r = tanhf(r);
      if (DACT) {
        const float a = act_in[(size_t)blockIdx.y * COUT * vol + c * vol + o];
        r *= (1.f - a * a);
      }
      ob[c * vol + o] = r;
    }
  }
}

// dW[co][ci][tap] += sum_b sum_p dz[b][co](p) * x[b][ci](p + tap)
template <int CIN, int COUT>
__global__ void __launch_bounds__(NTHR) k_conv_bwd_w(const float* __restrict__ x, const float* __restrict__ dz,
                                                     float* __restrict__ dw, Dims d, int nbatch) {
  extern __shared__ float sm[];
  float* xs = sm;            // [CIN][CS] halo tiles
  float* zs = sm + CIN * CS;  // [COUT][TZ][TY][TX]
  const int pair = threadIdx.x;
  const bool own = pair < CIN * COUT;
  const int co = own ? pair / CIN : 0, ci = own ? pair % CIN : 0;
  float acc[27];
#pragma unroll
  for (int k = 0; k < 27; ++k) acc[k] = 0.f;
  const size_t plane = (size_t)d.n1 * d.n2, vol = plane * d.n3;
  const int ntiles = d.tiles_x * d.tiles_y * d.tiles_z;
  for (long long w = blockIdx.x; w < (long long)ntiles * nbatch; w += gridDim.x) {
    const int b = (int)(w / ntiles), t = (int)(w % ntiles);
    const int bx = t % d.tiles_x, by = (t / d.tiles_x) % d.tiles_y, bz = t / (d.tiles_x * d.tiles_y);
    const int x0 = bx * TX, y0 = by * TY, z0 = bz * TZ;
    __syncthreads();
    load_tile<CIN>(xs, x + (size_t)b * CIN * vol, d, x0, y0, z0);
    for (int e = threadIdx.x; e < COUT * NTHR; e += NTHR) {
      const int p = e % NTHR, c = e / NTHR;
      const int px = x0 + p % TX, py = y0 + (p / TX) % TY, pz = z0 + p / (TX * TY);
      zs[e] = (px < d.n1 && py < d.n2 && pz < d.n3)
                  ? __ldg(dz + (size_t)b * COUT * vol + c * vol + (size_t)pz * plane + (size_t)py * d.n1 + px)
                  : 0.f;
    }
    __syncthreads();
    if (own) {
      for (int p = 0; p < NTHR; ++p) {
        const float g = zs[co * NTHR + p];
        const int px = p % TX, py = (p / TX) % TY, pz = p / (TX * TY);
#pragma unroll
        for (int kz = 0; kz < 3; ++kz)
#pragma unroll
          for (int ky = 0; ky < 3; ++ky)
#pragma unroll
            for (int kx = 0; kx < 3; ++kx)
              acc[(kz * 3 + ky) * 3 + kx] += g * xs[ci * CS + ((pz + kz) * HY + py + ky) * HX + px + kx];
      }
    }
  }
  if (own) {
#pragma unroll
    for (int k = 0; k < 27; ++k) atomicAdd(dw + (co * CIN + ci) * 27 + k, acc[k]);
  }
}

// transposed + flipped weights for the adjoint convolution: wt[ci][co][26-tap] = w[co][ci][tap]
__global__ void k_transpose_w(const float* __restrict__ w, __nv_bfloat16* __restrict__ wt, int cin, int cout) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cin * cout * 27; e += gridDim.x * blockDim.x) {
    const int tap = e % 27, ci = (e / 27) % cin, co = e / (27 * cin);
    wt[(ci * cout + co) * 27 + (26 - tap)] = __float2bfloat16(w[e]);
  }
}

// MSE over the interior (margin points from every face) of [batch][1][n3][n2][n1]
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy, Dims d,
                       int nbatch, int margin, double inv_count, double* loss) {
  const size_t vol = (size_t)d.n1 * d.n2 * d.n3;
  double s = 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol * nbatch; e += (size_t)gridDim.x * blockDim.x) {
    const size_t o = e % vol;
    const int x = (int)(o % d.n1), yy = (int)((o / d.n1) % d.n2), z = (int)(o / ((size_t)d.n1 * d.n2));
    const bool in = x >= margin && x < d.n1 - margin && yy >= margin && yy < d.n2 - margin && z >= margin &&
                    z < d.n3 - margin;
    const float diff = in ? y[e] - t[e] : 0.f;
    dy[e] = (float)(2.0 * diff * inv_count);
    s += (double)diff * diff;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_count);
}

__global__ void k_adam(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                       float* __restrict__ m, float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    const float nw = w[e] - upd;
    w[e] = nw;
    wb[e] = __float2bfloat16(nw);
  }
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) wb[e] = __float2bfloat16(w[e]);
}

// gather batch patches by index: dst[b] = src[idx[b]] (each patch `vol` floats)
__global__ void k_gather_patches(const float* __restrict__ src, const int* __restrict__ idx, float* __restrict__ dst,
                                 int nb, size_t vol) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol * nb; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = src[(size_t)idx[e / vol] * vol + e % vol];
}

// per-band RMS scaling for inference: s[b] = rms(g_b) (guarded), x = g/s
__global__ void k_rms(const float* __restrict__ g, double* __restrict__ s2, size_t vol) {
  double acc = 0.0;
  const float* gb = g + (size_t)blockIdx.y * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x)
    acc += (double)gb[e] * gb[e];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(s2 + blockIdx.y, acc);
}
// x = g * f per band (x may be g: in place)
__global__ void k_scale(const float* g, float* x, const double* __restrict__ s2, size_t vol, int inverse) {
  const double r = sqrt(s2[blockIdx.y] / (double)vol);
  const float f = r > 0.0 ? (float)(inverse ? r : 1.0 / r) : 0.f;
  const float* gb = g + (size_t)blockIdx.y * vol;
  float* xb = x + (size_t)blockIdx.y * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x)
    xb[e] = gb[e] * f;
}

// ---- training-pair harvest -------------------------------------------------------------
// per-band dot products out[b] += <a_b|b_b> (double accumulation)
__global__ void k_dot_bands(const float* __restrict__ a, const float* __restrict__ b, double* __restrict__ out,
                            size_t vol) {
  double acc = 0.0;
  const float* ab = a + (size_t)blockIdx.y * vol;
  const float* bb = b + (size_t)blockIdx.y * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x)
    acc += (double)ab[e] * bb[e];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out + blockIdx.y, acc);
}
// CG gradient of the band update, scaled to unit RMS: g = -2 (hx - E x), E = <x|hx>/<x|x>
// (the real-build gradient of src/conjugate_gradient/cg_module.f90:152); xx, xh, gg per band
__global__ void k_grad_bands(const float* __restrict__ x, const float* __restrict__ hx, float* __restrict__ g,
                             const double* __restrict__ xx, const double* __restrict__ xh, size_t vol) {
  const double E = xh[blockIdx.y] / xx[blockIdx.y];
  const size_t o = (size_t)blockIdx.y * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x)
    g[o + e] = (float)(-2.0 * ((double)hx[o + e] - E * (double)x[o + e]));
}
// r = sigma x - a ; p = r   (a = (T + sigma) y0 with y0 = x)
__global__ void k_tcg_init(const float* __restrict__ x, const float* __restrict__ a, float* __restrict__ r,
                           float* __restrict__ pp, float sigma, size_t n) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const float v = sigma * x[e] - a[e];
    r[e] = v;
    pp[e] = v;
  }
}
// y += alpha p ; r -= alpha ap ; alpha = rr / pap per band (skipped for converged bands)
__global__ void k_tcg_step(float* __restrict__ y, float* __restrict__ r, const float* __restrict__ pp,
                           const float* __restrict__ ap, const double* __restrict__ rr, const double* __restrict__ pap,
                           size_t vol) {
  const int b = blockIdx.y;
  if (!(pap[b] > 0.0) || !(rr[b] > 0.0)) return;
  const float al = (float)(rr[b] / pap[b]);
  const size_t o = (size_t)b * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x) {
    y[o + e] += al * pp[o + e];
    r[o + e] -= al * ap[o + e];
  }
}
// p = r + beta p ; beta = rrn / rr
__global__ void k_tcg_dir(float* __restrict__ pp, const float* __restrict__ r, const double* __restrict__ rr,
                          const double* __restrict__ rrn, size_t vol) {
  const int b = blockIdx.y;
  if (!(rr[b] > 0.0)) return;
  const float be = (float)(rrn[b] / rr[b]);
  const size_t o = (size_t)b * vol;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < vol; e += (size_t)gridDim.x * blockDim.x)
    pp[o + e] = r[o + e] + be * pp[o + e];
}
// copy pn^3 patches (periodic wrap) of x and t: spec = (band, x0, y0, z0)
__global__ void k_extract(const float* __restrict__ fx, const float* __restrict__ ft, const int4* __restrict__ spec,
                          float* __restrict__ dx, float* __restrict__ dt, int npatch, int pn, int n1, int n2, int n3) {
  const size_t pv = (size_t)pn * pn * pn, vol = (size_t)n1 * n2 * n3;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < pv * npatch; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e / pv);
    const int q = (int)(e % pv);
    const int4 sp = spec[i];
    const int x = (sp.y + q % pn) % n1, y = (sp.z + (q / pn) % pn) % n2, z = (sp.w + q / (pn * pn)) % n3;
    const size_t src = (size_t)sp.x * vol + ((size_t)z * n2 + y) * n1 + x;
    dx[e] = fx[src];
    dt[e] = ft[src];
  }
}

// ---- tensor-core inference path (full periodic grids) ----------------------------------
// Activations of a band: BF16 in two half-planes of 8 channels, [2][ng][8] (16 bytes per point
// per half), so that 8 consecutive points of one half form one 128-byte core matrix of the
// no-swizzle K-major UMMA layout.
constexpr int TC_TX = 32;                    // output x per tile
constexpr int TC_HX = TC_TX + 2;             // staged x (periodic halo)
constexpr int TC_TY = 11;                    // output rows per tile
constexpr int TC_HY = TC_TY + 2;
constexpr int TC_NM = (TC_TY * TC_HX + 127) / 128;  // M-tiles (128 rows) per output plane
constexpr int TC_PB = TC_NM * 128 + 2 * TC_HX + 2;  // staged points per plane (guards included)
constexpr int TC_SLOTS = 4;                  // plane ring
constexpr int TC_TZ = 16;                    // output planes per CTA
constexpr uint32_t TC_POLLS = 1u << 22;

__device__ __forceinline__ uint64_t umma_desc_nosw(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version (sm_100); layout bits 61-63 = 0: no swizzle
  return d;
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// UMMA B operands of one 16->16 layer: for each tap, [khalf][co 0..15][8 ci] BF16 from the FP32
// master weights w[co][ci][tap].
__global__ void k_tc_pack_w(const float* __restrict__ w, __nv_bfloat16* __restrict__ wp) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < 27 * 256; e += gridDim.x * blockDim.x) {
    const int i = e % 8, co = (e / 8) % 16, kh = (e / 128) % 2, tap = e / 256;
    wp[e] = __float2bfloat16(w[(co * 16 + kh * 8 + i) * 27 + tap]);
  }
}

__device__ __forceinline__ int wrapi(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ int wrap1(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }
// hardware tanh (sm_75+ instruction; relative error ~5e-4, below the BF16 rounding of the result)
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Layer 1 (1 -> 16, tanh) on CUDA cores: x = g / rms(g) read from the FP32 band, written as
// BF16 half-planes.  A thread owns 4 consecutive x points (n1 a multiple of 4).
__global__ void __launch_bounds__(256) k_tc_layer1(const float* __restrict__ g, const double* __restrict__ s2,
                                                   const __nv_bfloat16* __restrict__ w1, uint4* __restrict__ out,
                                                   int n1, int n2, int n3) {
  __shared__ float ws[27 * 16];  // [tap][co]
  for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x) ws[e] = __bfloat162float(w1[(e % 16) * 27 + e / 16]);
  __syncthreads();
  const size_t ng = (size_t)n1 * n2 * n3;
  const int b = blockIdx.y;
  const double rms = sqrt(s2[b] / (double)ng);
  const float sc = rms > 0.0 ? (float)(1.0 / rms) : 0.f;
  const float* gb = g + (size_t)b * ng;
  uint4* ob = out + (size_t)b * 2 * ng;
  const int q1 = n1 / 4;
  const size_t nq = ng / 4;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq; t += (size_t)gridDim.x * blockDim.x) {
    const int xq = (int)(t % q1), y = (int)((t / q1) % n2), z = (int)(t / ((size_t)q1 * n2));
    const int x0 = xq * 4;
    float acc[4][16];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[i][c] = 0.f;
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
      for (int ky = 0; ky < 3; ++ky) {
        const float* row = gb + ((size_t)wrap1(z + kz - 1, n3) * n2 + wrap1(y + ky - 1, n2)) * n1;
        float v[6];
        const float4 m = *reinterpret_cast<const float4*>(row + x0);
        v[0] = __ldg(row + wrap1(x0 - 1, n1));
        v[1] = m.x; v[2] = m.y; v[3] = m.z; v[4] = m.w;
        v[5] = __ldg(row + wrap1(x0 + 4, n1));
#pragma unroll
        for (int kx = 0; kx < 3; ++kx) {
          const float* wt = ws + ((kz * 3 + ky) * 3 + kx) * 16;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float xv = v[i + kx] * sc;
#pragma unroll
            for (int c = 0; c < 16; ++c) acc[i][c] = fmaf(wt[c], xv, acc[i][c]);
          }
        }
      }
    const size_t pt0 = ((size_t)z * n2 + y) * n1 + x0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      __align__(16) __nv_bfloat16 h[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) h[c] = __float2bfloat16(tanh_fast(acc[i][c]));
      ob[pt0 + i] = *reinterpret_cast<const uint4*>(h);
      ob[ng + pt0 + i] = *reinterpret_cast<const uint4*>(h + 8);
    }
  }
}

// Layer 4 (16 -> 1, linear) on CUDA cores from BF16 half-planes, times rms(g): the
// preconditioned band.  A thread owns 4 consecutive x points.
__global__ void __launch_bounds__(256) k_tc_layer4(const uint4* __restrict__ in, const double* __restrict__ s2,
                                                   const __nv_bfloat16* __restrict__ w4, float* __restrict__ pg,
                                                   int n1, int n2, int n3) {
  __shared__ float ws[27 * 16];  // [tap][ci]
  for (int e = threadIdx.x; e < 27 * 16; e += blockDim.x) ws[e] = __bfloat162float(w4[(e % 16) * 27 + e / 16]);
  __syncthreads();
  const size_t ng = (size_t)n1 * n2 * n3;
  const int b = blockIdx.y;
  const float rms = (float)sqrt(s2[b] / (double)ng);
  const uint4* ib = in + (size_t)b * 2 * ng;
  const int q1 = n1 / 4;
  const size_t nq = ng / 4;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nq; t += (size_t)gridDim.x * blockDim.x) {
    const int xq = (int)(t % q1), y = (int)((t / q1) % n2), z = (int)(t / ((size_t)q1 * n2));
    const int x0 = xq * 4;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kz = 0; kz < 3; ++kz)
#pragma unroll
      for (int ky = 0; ky < 3; ++ky) {
        const size_t rb = ((size_t)wrap1(z + kz - 1, n3) * n2 + wrap1(y + ky - 1, n2)) * n1;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const uint4* row = ib + (size_t)hh * ng + rb;
#pragma unroll
          for (int j = 0; j < 6; ++j) {
            const int xx = j == 0 ? wrap1(x0 - 1, n1) : (j == 5 ? wrap1(x0 + 4, n1) : x0 + j - 1);
            const uint4 u = __ldg(row + xx);
            const __nv_bfloat16* hv = reinterpret_cast<const __nv_bfloat16*>(&u);
            float a8[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) a8[c] = __bfloat162float(hv[c]);
#pragma unroll
            for (int kx = 0; kx < 3; ++kx) {
              const int i = j - kx;  // output point fed by input j through tap kx
              if (i >= 0 && i < 4) {
                const float* wt = ws + ((kz * 3 + ky) * 3 + kx) * 16 + hh * 8;
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[i] = fmaf(wt[c], a8[c], acc[i]);
              }
            }
          }
        }
      }
    *reinterpret_cast<float4*>(pg + (size_t)b * ng + ((size_t)z * n2 + y) * n1 + x0) =
        make_float4(acc[0] * rms, acc[1] * rms, acc[2] * rms, acc[3] * rms);
  }
}

// Layers 2 and 3 (16 -> 16, tanh) on the tensor cores.  A CTA (4 warps) owns a 32 x 11 output
// tile of x-rows over TC_TZ planes of one band.  Input planes (with a one-point periodic halo)
// arrive by bulk copies (TMA engine; contiguous row pieces in the half-plane layout) in a ring
// of TC_SLOTS planes; for output plane z each of the 27 taps is one tcgen05.mma per 128-row
// M-tile whose A descriptor is the staged plane z + dz shifted by dy rows and dx points (rows of
// an M-tile are consecutive staged positions, so the two halo columns of every row produce
// outputs that are discarded), B the tap's 16 x 16 weights, D an FP32 accumulator of 16 TMEM
// columns.  Two accumulator sets let the MMAs of plane z+1 run during the epilogue (tanh,
// BF16 half-planes) of plane z.  All waits are bounded; a timeout sets *status and every copy
// in flight is waited for before the CTA exits.
__global__ void __launch_bounds__(128) k_tc_mid(const uint4* __restrict__ in, const __nv_bfloat16* __restrict__ wp,
                                                uint4* __restrict__ out, int n1, int n2, int n3, int tiles_x,
                                                int tiles_y, int tiles_z, unsigned* status) {
  extern __shared__ __align__(128) unsigned char tsm[];
  constexpr int PLANE_BYTES = 2 * TC_PB * 16;
  constexpr uint32_t STAGED_BYTES = 2u * TC_HY * TC_HX * 16u;
  unsigned char* ring = tsm;                                   // [slot][half][TC_PB][16 B]
  unsigned char* wsm = tsm + TC_SLOTS * PLANE_BYTES;           // [27][2][16][16 B]
  uint64_t* full = reinterpret_cast<uint64_t*>(wsm + 27 * 512);  // [TC_SLOTS]
  uint64_t* done = full + TC_SLOTS;                              // [2]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const size_t ng = (size_t)n1 * n2 * n3;
  int t = blockIdx.x;
  const int bx = t % tiles_x;
  t /= tiles_x;
  const int by = t % tiles_y;
  t /= tiles_y;
  const int bz = t % tiles_z;
  const int band = blockIdx.y;
  const int x0 = bx * TC_TX, y0 = by * TC_TY, z0 = bz * TC_TZ;
  const int zend = min(z0 + TC_TZ, n3);
  const int nplanes = zend - z0 + 2;  // staged planes z0-1 .. zend
  const uint4* ib = in + (size_t)band * 2 * ng;
  uint4* ob = out + (size_t)band * 2 * ng;

  for (int e = tid; e < 27 * 32; e += 128)
    reinterpret_cast<uint4*>(wsm)[e] = __ldg(reinterpret_cast<const uint4*>(wp) + e);
  if (tid == 0) {
    for (int i = 0; i < TC_SLOTS; ++i) mbar_init(&full[i], 1);
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(128u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_proxy_async_smem();  // the weights were written through the generic proxy
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  // thread 0: bulk-copy staged plane i (= z0 - 1 + i) into ring slot i % TC_SLOTS; position
  // 1 + r * TC_HX + c holds point (x0 - 1 + c, y0 - 1 + r), copied as contiguous x pieces
  int issued = 0;
  auto issue_plane = [&]() {
    const int i = issued++;
    const int slot = i % TC_SLOTS;
    unsigned char* pb = ring + (size_t)slot * PLANE_BYTES;
    const int zg = wrapi(z0 - 1 + i, n3);
    mbar_arrive_expect_tx(&full[slot], STAGED_BYTES);
    for (int hh = 0; hh < 2; ++hh)
      for (int r = 0; r < TC_HY; ++r) {
        const int gy = wrapi(y0 - 1 + r, n2);
        const uint4* src = ib + (size_t)hh * ng + ((size_t)zg * n2 + gy) * n1;
        unsigned char* dst = pb + ((size_t)hh * TC_PB + 1 + (size_t)r * TC_HX) * 16;
        int c = 0;
        while (c < TC_HX) {
          const int gx = wrapi(x0 - 1 + c, n1);
          const int len = min(TC_HX - c, n1 - gx);
          bulk_g2s(dst + (size_t)c * 16, src + gx, (uint32_t)len * 16u, &full[slot]);
          c += len;
        }
      }
  };
  int landed = 0;  // thread 0: planes 0 .. landed-1 have been observed complete (waited in order)
  auto plane_ready = [&](int i) {
    const bool r = mbar_wait_bounded(&full[i % TC_SLOTS], (uint32_t)((i / TC_SLOTS) & 1), TC_POLLS);
    if (r) landed = i + 1;
    return r;
  };
  // M = 128, N = 16, BF16 x BF16 -> FP32, both K-major
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(16 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
  // Descriptors are built once: a tap only moves the start address (16-byte units, one point
  // of a half-plane), which the descriptor holds in its low 14 bits; every shared address here
  // is below 2^18 bytes, so the additions never carry out of that field.
  const uint64_t dring = umma_desc_nosw(smem_u32(ring), TC_PB * 16, 128);
  const uint64_t dwts = umma_desc_nosw(smem_u32(wsm), 256, 128);
  auto issue_mma = [&](int z) {  // thread 0; planes z-1, z, z+1 ready
    const int buf = (z - z0) & 1;
    const int s0 = (z - z0) % TC_SLOTS;  // slot of plane z - 1
    uint64_t dpl[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) dpl[d] = dring + (uint64_t)(((s0 + d) % TC_SLOTS) * (PLANE_BYTES >> 4));
#pragma unroll
    for (int mt = 0; mt < TC_NM; ++mt) {
#pragma unroll
      for (int tap = 0; tap < 27; ++tap) {
        const int dz = tap / 9, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        const int row0 = 1 + TC_HX + mt * 128 + dy * TC_HX + dx;  // staged position of M row 0
        umma_bf16(tmem + (uint32_t)(buf * 64 + mt * 16), dpl[dz] + (uint64_t)row0, dwts + (uint64_t)(tap * 32),
                  idesc, tap > 0 ? 1u : 0u);
      }
    }
    umma_commit(&done[buf]);
  };
  int mma_issued = 0, mma_waited = 0;  // thread 0: MMA groups committed / observed complete

  bool ok = true;
  if (tid == 0) {
    for (int i = 0; i < TC_SLOTS && i < nplanes; ++i) issue_plane();
    ok = plane_ready(0) && plane_ready(1) && plane_ready(2);
    tc_fence_after();
    if (ok) {
      issue_mma(z0);
      ++mma_issued;
    }
  }
  for (int z = z0; z < zend; ++z) {
    const int rel = z - z0;
    if (tid == 0 && ok && z + 1 < zend) {
      ok = plane_ready(rel + 3);  // plane z + 2 (issued while earlier planes were computed)
      if (ok) {
        issue_mma(z + 1);
        ++mma_issued;
      }
    }
    const bool waited = mbar_wait_bounded(&done[rel & 1], (uint32_t)((rel >> 1) & 1), TC_POLLS);
    if (waited && tid == 0) mma_waited = rel + 1;
    tc_fence_after();
    if (waited && ok) {
      // the MMAs of plane z have read plane z - 1: its slot takes plane z + 3
      if (tid == 0 && issued < nplanes) issue_plane();
#pragma unroll 1
      for (int mt = 0; mt < TC_NM; ++mt) {
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((rel & 1) * 64 + mt * 16), v);
        const int e = mt * 128 + warp * 32 + lane;  // output position from row 1, column 0
        const int r = e / TC_HX, cx = e % TC_HX;
        const int gx = x0 - 1 + cx, gy = y0 + r;
        if (r < TC_TY && cx >= 1 && cx <= TC_TX && gx < n1 && gy < n2) {
          __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
          for (int cc = 0; cc < 16; ++cc) hb[cc] = __float2bfloat16(tanh_fast(v[cc]));
          const size_t pt = ((size_t)z * n2 + gy) * n1 + gx;
          ob[pt] = *reinterpret_cast<const uint4*>(hb);
          ob[ng + pt] = *reinterpret_cast<const uint4*>(hb + 8);
        }
      }
    }
    tc_fence_before();
    // all reads of this accumulator set are done before the MMAs of plane z + 2 reuse it
    const int bad = __syncthreads_or(!(waited && ok));
    tc_fence_after();
    if (bad) {
      ok = false;
      break;
    }
  }
  if (tid == 0) {
    if (!ok) atomicOr(status, DEV_WAIT_TIMEOUT);
    // copies in flight and committed MMAs complete before the shared memory is released
    // (only those not yet observed: a slot's barrier has moved on past the earlier phases)
    bool drained = true;
    for (int i = landed; i < issued; ++i) drained = plane_ready(i) && drained;
    for (int m = mma_waited; m < mma_issued; ++m)
      drained = mbar_wait_bounded(&done[m & 1], (uint32_t)((m >> 1) & 1), TC_POLLS) && drained;
    if (!drained) atomicOr(status, DEV_WAIT_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(128u));
}

}  // namespace lpc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct LpcState {
  DBuf w, wb, wt, dw, m, v;   // FP32 master, BF16 copy, BF16 transposed, grads, Adam moments
  DBuf tcw, tca;              // tensor-core path: packed layer-2/3 weights, BF16 activations
  DBuf act, dact, batch_x, batch_t, dy, idx, loss, s2;
  DBuf set_x, set_t;          // training set: [capacity][pn^3] inputs and targets
  DBuf hv, hs;                // harvest work fields / per-band scalars
  DBuf io_a, io_b;            // staging for host-pointer calls
  int set_cap = 0, set_n = 0, set_pn = 0;
  bool ready = false;
  long long steps = 0;
};
static LpcState g_lpc;

static lpc::Dims make_dims(int n1, int n2, int n3, int periodic) {
  lpc::Dims d;
  d.n1 = n1; d.n2 = n2; d.n3 = n3; d.periodic = periodic;
  d.tiles_x = (n1 + lpc::TX - 1) / lpc::TX;
  d.tiles_y = (n2 + lpc::TY - 1) / lpc::TY;
  d.tiles_z = (n3 + lpc::TZ - 1) / lpc::TZ;
  return d;
}

template <int CIN, int COUT, bool ACT, bool DACT>
static int conv_fwd(Ctx& c, const float* in, const __nv_bfloat16* w, float* out, const float* act, const lpc::Dims& d,
                    int nbatch) {
  if constexpr (COUT % 2 == 0) {
    constexpr int CC = CIN < lpc::FCC ? CIN : lpc::FCC;
    const size_t smem = sizeof(float) * (CC * 27 * COUT + CC * lpc::FCS);
    auto kern = lpc::k_conv_fwd4<CIN, COUT, ACT, DACT>;
    static bool attr4 = false;
    if (!attr4) {
      RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr4 = true;
    }
    const int tx = (d.n1 + lpc::FX - 1) / lpc::FX, ty = (d.n2 + lpc::FY - 1) / lpc::FY;
    const int tz = (d.n3 + lpc::FZ - 1) / lpc::FZ;
    dim3 grid(tx * ty * tz, nbatch);
    kern<<<grid, 256, smem, c.stream>>>(in, w, out, act, d, tx, ty);
    c.launches++;
    return check_launch("lpc_conv_fwd");
  }
  const size_t smem = sizeof(float) * (COUT * CIN * 27 + CIN * lpc::CS);
  auto kern = lpc::k_conv_fwd<CIN, COUT, ACT, DACT>;
  static bool attr = false;
  if (!attr) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  dim3 grid(d.tiles_x * d.tiles_y * d.tiles_z, nbatch);
  kern<<<grid, lpc::NTHR, smem, c.stream>>>(in, w, out, act, d);
  c.launches++;
  return check_launch("lpc_conv_fwd");
}

template <int CIN, int COUT>
static int conv_bwd_w(Ctx& c, const float* x, const float* dz, float* dw, const lpc::Dims& d, int nbatch) {
  const size_t smem = sizeof(float) * (CIN * lpc::CS + COUT * lpc::NTHR);
  auto kern = lpc::k_conv_bwd_w<CIN, COUT>;
  static bool attr = false;
  if (!attr) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  kern<<<2 * 148, lpc::NTHR, smem, c.stream>>>(x, dz, dw, d, nbatch);
  c.launches++;
  return check_launch("lpc_conv_bwd_w");
}

static int lpc_alloc(Ctx& c) {
  (void)c;
  RS_TRY(g_lpc.w.ensure(sizeof(float) * lpc::WTOT));
  RS_TRY(g_lpc.wb.ensure(sizeof(__nv_bfloat16) * lpc::WTOT));
  RS_TRY(g_lpc.wt.ensure(sizeof(__nv_bfloat16) * lpc::WTOT));
  RS_TRY(g_lpc.dw.ensure(sizeof(float) * lpc::WTOT));
  RS_TRY(g_lpc.m.ensure(sizeof(float) * lpc::WTOT));
  RS_TRY(g_lpc.v.ensure(sizeof(float) * lpc::WTOT));
  RS_TRY(g_lpc.loss.ensure(sizeof(double) * 4));
  return 0;
}

// forward through the 4 layers; act: 3 activation buffers of [nb][16][vol] each
static int forward(Ctx& c, const float* x, float* y, float* act, const lpc::Dims& d, int nb) {
  const size_t vol = (size_t)d.n1 * d.n2 * d.n3;
  const __nv_bfloat16* wb = g_lpc.wb.as<__nv_bfloat16>();
  float* a1 = act;
  float* a2 = a1 + (size_t)nb * 16 * vol;
  float* a3 = a2 + (size_t)nb * 16 * vol;
  RS_TRY((conv_fwd<1, 16, true, false>(c, x, wb + lpc::woff(0), a1, nullptr, d, nb)));
  RS_TRY((conv_fwd<16, 16, true, false>(c, a1, wb + lpc::woff(1), a2, nullptr, d, nb)));
  RS_TRY((conv_fwd<16, 16, true, false>(c, a2, wb + lpc::woff(2), a3, nullptr, d, nb)));
  RS_TRY((conv_fwd<16, 1, false, false>(c, a3, wb + lpc::woff(3), y, nullptr, d, nb)));
  return 0;
}

// loss gradient dW for a batch (x, dy given); act holds the forward activations
static int backward(Ctx& c, const float* x, const float* dy, const float* act, float* dact, const lpc::Dims& d, int nb) {
  const size_t vol = (size_t)d.n1 * d.n2 * d.n3;
  const float* a1 = act;
  const float* a2 = a1 + (size_t)nb * 16 * vol;
  const float* a3 = a2 + (size_t)nb * 16 * vol;
  float* dA = dact;
  float* dB = dact + (size_t)nb * 16 * vol;
  float* dw = g_lpc.dw.as<float>();
  __nv_bfloat16* wt = g_lpc.wt.as<__nv_bfloat16>();
  const float* w = g_lpc.w.as<float>();
  for (int l = 0; l < lpc::NL; ++l)
    lpc::k_transpose_w<<<16, 256, 0, c.stream>>>(w + lpc::woff(l), wt + lpc::woff(l), lpc::CH[l], lpc::CH[l + 1]);
  c.launches += lpc::NL;
  // layer 4 (16 -> 1, linear)
  RS_TRY((conv_bwd_w<16, 1>(c, a3, dy, dw + lpc::woff(3), d, nb)));
  RS_TRY((conv_fwd<1, 16, false, true>(c, dy, wt + lpc::woff(3), dA, a3, d, nb)));  // dz3
  // layer 3
  RS_TRY((conv_bwd_w<16, 16>(c, a2, dA, dw + lpc::woff(2), d, nb)));
  RS_TRY((conv_fwd<16, 16, false, true>(c, dA, wt + lpc::woff(2), dB, a2, d, nb)));  // dz2
  // layer 2
  RS_TRY((conv_bwd_w<16, 16>(c, a1, dB, dw + lpc::woff(1), d, nb)));
  RS_TRY((conv_fwd<16, 16, false, true>(c, dB, wt + lpc::woff(1), dA, a1, d, nb)));  // dz1
  // layer 1
  RS_TRY((conv_bwd_w<1, 16>(c, x, dA, dw + lpc::woff(0), d, nb)));
  return 0;
}

int lpc_init_weights(Ctx& c, uint64_t seed) {
  RS_TRY(lpc_alloc(c));
  std::vector<float> w(lpc::WTOT);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < lpc::NL; ++l) {
    std::normal_distribution<double> nd(0.0, 1.0 / std::sqrt(27.0 * lpc::CH[l]));
    for (int e = 0; e < 27 * lpc::CH[l] * lpc::CH[l + 1]; ++e) w[lpc::woff(l) + e] = (float)nd(rng);
  }
  RS_CUDA(cudaMemcpy(g_lpc.w.p, w.data(), sizeof(float) * lpc::WTOT, cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemsetAsync(g_lpc.m.p, 0, sizeof(float) * lpc::WTOT, c.stream));
  RS_CUDA(cudaMemsetAsync(g_lpc.v.p, 0, sizeof(float) * lpc::WTOT, c.stream));
  lpc::k_to_bf16<<<32, 256, 0, c.stream>>>(g_lpc.w.as<float>(), g_lpc.wb.as<__nv_bfloat16>(), lpc::WTOT);
  c.launches++;
  g_lpc.ready = true;
  g_lpc.steps = 0;
  return check_launch("lpc_init");
}

int lpc_set_weights(Ctx& c, const float* w) {
  RS_TRY(lpc_alloc(c));
  RS_CUDA(cudaMemcpy(g_lpc.w.p, w, sizeof(float) * lpc::WTOT, cudaMemcpyHostToDevice));
  lpc::k_to_bf16<<<32, 256, 0, c.stream>>>(g_lpc.w.as<float>(), g_lpc.wb.as<__nv_bfloat16>(), lpc::WTOT);
  c.launches++;
  RS_CUDA(cudaMemsetAsync(g_lpc.m.p, 0, sizeof(float) * lpc::WTOT, c.stream));
  RS_CUDA(cudaMemsetAsync(g_lpc.v.p, 0, sizeof(float) * lpc::WTOT, c.stream));
  g_lpc.ready = true;
  g_lpc.steps = 0;
  return check_launch("lpc_set_weights");
}

int lpc_get_weights(Ctx& c, float* w) {
  RS_CHECK(g_lpc.ready, RSDFT_ERR_STATE, "learned preconditioner not initialised");
  RS_CUDA(cudaMemcpyAsync(w, g_lpc.w.p, sizeof(float) * lpc::WTOT, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

// network output for nb fields of n1 x n2 x n3 (device pointers, no input scaling)
int lpc_forward(Ctx& c, const float* x, float* y, int nb, int n1, int n2, int n3, int periodic) {
  RS_CHECK(g_lpc.ready, RSDFT_ERR_STATE, "learned preconditioner not initialised");
  const lpc::Dims d = make_dims(n1, n2, n3, periodic);
  const size_t vol = (size_t)n1 * n2 * n3;
  RS_TRY(g_lpc.act.ensure(sizeof(float) * 3 * 16 * vol * nb));
  return forward(c, x, y, g_lpc.act.as<float>(), d, nb);
}

// loss and dL/dW (host) for a batch of patches (device x, t)
int lpc_loss_grad(Ctx& c, const float* x, const float* t, int nb, int n, int margin, double* loss, float* grad) {
  RS_CHECK(g_lpc.ready, RSDFT_ERR_STATE, "learned preconditioner not initialised");
  const lpc::Dims d = make_dims(n, n, n, 0);
  const size_t vol = (size_t)n * n * n;
  const int inner = n - 2 * margin;
  RS_CHECK(inner > 0, RSDFT_ERR_ARG, "margin %d too large for patches of %d", margin, n);
  RS_TRY(g_lpc.act.ensure(sizeof(float) * 3 * 16 * vol * nb));
  RS_TRY(g_lpc.dact.ensure(sizeof(float) * 2 * 16 * vol * nb));
  RS_TRY(g_lpc.dy.ensure(sizeof(float) * 2 * vol * nb));
  float* y = g_lpc.dy.as<float>();
  float* dy = y + vol * nb;
  RS_TRY(forward(c, x, y, g_lpc.act.as<float>(), d, nb));
  RS_CUDA(cudaMemsetAsync(g_lpc.loss.p, 0, sizeof(double), c.stream));
  const double inv = 1.0 / ((double)inner * inner * inner * nb);
  lpc::k_loss<<<4 * 148, 256, 0, c.stream>>>(y, t, dy, d, nb, margin, inv, g_lpc.loss.as<double>());
  c.launches++;
  RS_CUDA(cudaMemsetAsync(g_lpc.dw.p, 0, sizeof(float) * lpc::WTOT, c.stream));
  RS_TRY(backward(c, x, dy, g_lpc.act.as<float>(), g_lpc.dact.as<float>(), d, nb));
  if (loss) RS_CUDA(cudaMemcpyAsync(loss, g_lpc.loss.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  if (grad) RS_CUDA(cudaMemcpyAsync(grad, g_lpc.dw.p, sizeof(float) * lpc::WTOT, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return check_launch("lpc_loss_grad");
}

// Adam training on npatch (x, t) patches of n^3 (device pointers); loss per epoch to losses
int lpc_train(Ctx& c, const float* x, const float* t, int npatch, int n, int margin, int epochs, int batch,
              double lr, uint64_t seed, double* losses) {
  RS_CHECK(g_lpc.ready, RSDFT_ERR_STATE, "learned preconditioner not initialised");
  RS_CHECK(npatch > 0 && batch > 0 && epochs > 0 && n > 2 * margin, RSDFT_ERR_ARG, "bad training arguments");
  batch = std::min(batch, npatch);
  const lpc::Dims d = make_dims(n, n, n, 0);
  const size_t vol = (size_t)n * n * n;
  const int inner = n - 2 * margin;
  RS_TRY(g_lpc.act.ensure(sizeof(float) * 3 * 16 * vol * batch));
  RS_TRY(g_lpc.dact.ensure(sizeof(float) * 2 * 16 * vol * batch));
  RS_TRY(g_lpc.dy.ensure(sizeof(float) * 2 * vol * batch));
  RS_TRY(g_lpc.batch_x.ensure(sizeof(float) * 2 * vol * batch));
  RS_TRY(g_lpc.idx.ensure(sizeof(int) * (size_t)npatch));
  float* bx = g_lpc.batch_x.as<float>();
  float* bt = bx + vol * batch;
  float* y = g_lpc.dy.as<float>();
  float* dy = y + vol * batch;
  std::vector<int> order(npatch);
  for (int i = 0; i < npatch; ++i) order[i] = i;
  std::mt19937_64 rng(seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const double inv = 1.0 / ((double)inner * inner * inner * batch);
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    RS_CUDA(cudaMemcpyAsync(g_lpc.idx.p, order.data(), sizeof(int) * npatch, cudaMemcpyHostToDevice, c.stream));
    RS_CUDA(cudaMemsetAsync(g_lpc.loss.p, 0, sizeof(double), c.stream));
    const int nbt = npatch / batch;
    for (int bi = 0; bi < nbt; ++bi) {
      const int* ib = g_lpc.idx.as<int>() + (size_t)bi * batch;
      lpc::k_gather_patches<<<4 * 148, 256, 0, c.stream>>>(x, ib, bx, batch, vol);
      lpc::k_gather_patches<<<4 * 148, 256, 0, c.stream>>>(t, ib, bt, batch, vol);
      c.launches += 2;
      RS_TRY(forward(c, bx, y, g_lpc.act.as<float>(), d, batch));
      lpc::k_loss<<<4 * 148, 256, 0, c.stream>>>(y, bt, dy, d, batch, margin, inv, g_lpc.loss.as<double>());
      c.launches++;
      RS_CUDA(cudaMemsetAsync(g_lpc.dw.p, 0, sizeof(float) * lpc::WTOT, c.stream));
      RS_TRY(backward(c, bx, dy, g_lpc.act.as<float>(), g_lpc.dact.as<float>(), d, batch));
      g_lpc.steps++;
      const float c1 = 1.f - std::pow(b1, (float)g_lpc.steps), c2 = 1.f - std::pow(b2, (float)g_lpc.steps);
      lpc::k_adam<<<32, 256, 0, c.stream>>>(g_lpc.w.as<float>(), g_lpc.wb.as<__nv_bfloat16>(), g_lpc.dw.as<float>(),
                                            g_lpc.m.as<float>(), g_lpc.v.as<float>(), lpc::WTOT, (float)lr, b1, b2,
                                            eps, c1, c2);
      c.launches++;
      RS_TRY(check_launch("lpc_train"));
    }
    double l = 0.0;
    RS_CUDA(cudaMemcpyAsync(&l, g_lpc.loss.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    if (losses) losses[ep] = l / std::max(1, nbt);
  }
  return 0;
}

// Preconditioner application on full periodic grids: pg_b = rms(g_b) f(g_b / rms(g_b)).
// g, pg: nb bands of ng FP32 values (real build).
// Preconditioner application with the two 16 -> 16 layers on the tensor cores (BF16
// activations, FP32 accumulation in TMEM) and the thin first and last layers on CUDA cores.
static int lpc_apply_tc(Ctx& c, const float* g, float* pg, int nb) {
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  const size_t ng = c.ng;
  const int nbc = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)(8ull << 30) / (64 * ng)));
  RS_TRY(g_lpc.tcw.ensure(sizeof(__nv_bfloat16) * 2 * 27 * 256));
  RS_TRY(g_lpc.tca.ensure((size_t)64 * ng * nbc));
  RS_TRY(g_lpc.s2.ensure(sizeof(double) * nbc));
  __nv_bfloat16* w2 = g_lpc.tcw.as<__nv_bfloat16>();
  __nv_bfloat16* w3 = w2 + 27 * 256;
  lpc::k_tc_pack_w<<<27, 256, 0, c.stream>>>(g_lpc.w.as<float>() + lpc::woff(1), w2);
  lpc::k_tc_pack_w<<<27, 256, 0, c.stream>>>(g_lpc.w.as<float>() + lpc::woff(2), w3);
  c.launches += 2;
  constexpr size_t smem = (size_t)lpc::TC_SLOTS * 2 * lpc::TC_PB * 16 + 27 * 512 + 8 * (lpc::TC_SLOTS + 2) + 16;
  static bool attr = false;
  if (!attr) {
    RS_CUDA(cudaFuncSetAttribute(lpc::k_tc_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const int tx = (n1 + lpc::TC_TX - 1) / lpc::TC_TX, ty = (n2 + lpc::TC_TY - 1) / lpc::TC_TY;
  const int tz = (n3 + lpc::TC_TZ - 1) / lpc::TC_TZ;
  uint4* A = g_lpc.tca.as<uint4>();
  uint4* B = A + 2 * ng * nbc;
  const __nv_bfloat16* wb = g_lpc.wb.as<__nv_bfloat16>();
  ProfScope ps(c, "lpc", 0.0, 2.0 * 27 * (16 + 256 + 256 + 16) * (double)ng * nb);
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int nn = std::min(nbc, nb - b0);
    RS_CUDA(cudaMemsetAsync(g_lpc.s2.p, 0, sizeof(double) * nn, c.stream));
    lpc::k_rms<<<dim3(64, nn), 256, 0, c.stream>>>(g + (size_t)b0 * ng, g_lpc.s2.as<double>(), ng);
    const unsigned pblk = (unsigned)std::min<size_t>((ng / 4 + 255) / 256, 8 * 148);
    const double pts = (double)ng * nn;
    {
      ProfScope pl(c, "lpc_layer1", 36.0 * pts, 2.0 * 27 * 16 * pts);
      lpc::k_tc_layer1<<<dim3(pblk, nn), 256, 0, c.stream>>>(g + (size_t)b0 * ng, g_lpc.s2.as<double>(),
                                                              wb + lpc::woff(0), A, n1, n2, n3);
    }
    {
      ProfScope pl(c, "lpc_mid", 2 * 64.0 * pts, 2 * 2.0 * 27 * 256 * pts);
      lpc::k_tc_mid<<<dim3(tx * ty * tz, nn), 128, smem, c.stream>>>(A, w2, B, n1, n2, n3, tx, ty, tz, c.d_status);
      lpc::k_tc_mid<<<dim3(tx * ty * tz, nn), 128, smem, c.stream>>>(B, w3, A, n1, n2, n3, tx, ty, tz, c.d_status);
    }
    {
      ProfScope pl(c, "lpc_layer4", 36.0 * pts, 2.0 * 27 * 16 * pts);
      lpc::k_tc_layer4<<<dim3(pblk, nn), 256, 0, c.stream>>>(A, g_lpc.s2.as<double>(), wb + lpc::woff(3),
                                                              pg + (size_t)b0 * ng, n1, n2, n3);
    }
    c.launches += 5;
  }
  return check_launch("lpc_apply_tc");
}

int lpc_apply(Ctx& c, const float* g, float* pg, int nb) {
  RS_CHECK(g_lpc.ready, RSDFT_ERR_STATE, "learned preconditioner not initialised");
  if (c.lpc_fp32 == 0 && c.p.n1 % 4 == 0) return lpc_apply_tc(c, g, pg, nb);
  const lpc::Dims d = make_dims(c.p.n1, c.p.n2, c.p.n3, 1);
  const size_t vol = c.ng;
  // band chunk so that activations stay within ~2 GiB
  int nbc = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)(2u << 30) / (sizeof(float) * 50 * vol)));
  RS_TRY(g_lpc.act.ensure(sizeof(float) * 3 * 16 * vol * nbc));
  RS_TRY(g_lpc.batch_x.ensure(sizeof(float) * 2 * vol * nbc));
  RS_TRY(g_lpc.s2.ensure(sizeof(double) * nbc));
  ProfScope ps(c, "lpc", 0.0, 2.0 * 27 * (16 + 256 + 256 + 16) * (double)vol * nb);
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int nn = std::min(nbc, nb - b0);
    float* xs = g_lpc.batch_x.as<float>();
    float* ys = xs + vol * nbc;
    RS_CUDA(cudaMemsetAsync(g_lpc.s2.p, 0, sizeof(double) * nn, c.stream));
    lpc::k_rms<<<dim3(64, nn), 256, 0, c.stream>>>(g + (size_t)b0 * vol, g_lpc.s2.as<double>(), vol);
    lpc::k_scale<<<dim3(64, nn), 256, 0, c.stream>>>(g + (size_t)b0 * vol, xs, g_lpc.s2.as<double>(), vol, 0);
    c.launches += 2;
    RS_TRY(forward(c, xs, ys, g_lpc.act.as<float>(), d, nn));
    lpc::k_scale<<<dim3(64, nn), 256, 0, c.stream>>>(ys, pg + (size_t)b0 * vol, g_lpc.s2.as<double>(), vol, 1);
    c.launches++;
  }
  return check_launch("lpc_apply");
}

// Empty training set of `capacity` patch pairs of pn^3 points.
int lpc_dataset(Ctx& c, int capacity, int pn) {
  (void)c;
  RS_CHECK(capacity > 0 && pn >= 4 && pn <= 64, RSDFT_ERR_ARG, "bad training-set shape (%d patches of %d^3)", capacity,
           pn);
  const size_t pv = (size_t)pn * pn * pn;
  RS_TRY(g_lpc.set_x.ensure(sizeof(float) * pv * capacity));
  RS_TRY(g_lpc.set_t.ensure(sizeof(float) * pv * capacity));
  g_lpc.set_cap = capacity;
  g_lpc.set_n = 0;
  g_lpc.set_pn = pn;
  return 0;
}

// Append up to npatch (input, target) patch pairs taken from the resident bands of (k, s):
// input  = the CG gradient g_b = -2 (H psi_b - E_b psi_b) scaled to unit RMS,
// target = sigma (T + sigma)^-1 g_b, the screened-kinetic correction, solved by `iters` CG
//          steps on the finite-difference kinetic operator T of the Hamiltonian.
// Patches are cut at random corners (periodic wrap) from random bands.
int lpc_harvest(Ctx& c, int k, int s, int npatch, double sigma, int iters, uint64_t seed, int* added) {
  RS_CHECK(g_lpc.set_cap > 0, RSDFT_ERR_STATE, "no training set: call lpc_dataset first");
  RS_CHECK(!c.cplx, RSDFT_ERR_UNSUPPORTED, "the learned preconditioner is built for the real Gamma build");
  RS_CHECK(sigma > 0.0 && iters > 0, RSDFT_ERR_ARG, "sigma and iters must be positive");
  WaveFns& w = c.wfn(k, s);
  RS_CHECK(w.valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k + 1, s + 1);
  const int nb = c.kp[k].nband;
  const size_t vol = c.ng;
  npatch = std::min(npatch, g_lpc.set_cap - g_lpc.set_n);
  if (added) *added = 0;
  if (npatch <= 0) return 0;
  const int pn = g_lpc.set_pn;
  RS_CHECK(pn <= c.p.n1 && pn <= c.p.n2 && pn <= c.p.n3, RSDFT_ERR_ARG, "patch %d larger than the grid", pn);
  // band chunk: 6 FP32 fields per band within ~3 GiB
  const int nbc = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)(3u << 30) / (sizeof(float) * 6 * vol)));
  RS_TRY(g_lpc.hv.ensure(sizeof(float) * 6 * vol * nbc));
  RS_TRY(g_lpc.hs.ensure(sizeof(double) * 4 * nbc + sizeof(int4) * (size_t)npatch));
  float* X = g_lpc.hv.as<float>();
  float* HX = X + vol * nbc;
  float* G = HX + vol * nbc;
  float* Y = G + vol * nbc;
  float* R = Y + vol * nbc;
  float* P = R + vol * nbc;
  double* d1 = g_lpc.hs.as<double>();
  double* d2 = d1 + nbc;
  double* d3 = d2 + nbc;
  int4* spec = reinterpret_cast<int4*>(d1 + 4 * nbc);
  std::mt19937_64 rng(seed);
  const size_t pv = (size_t)pn * pn * pn;
  // patches per chunk in proportion to its bands
  int done = 0;
  for (int b0 = 0; b0 < nb && done < npatch; b0 += nbc) {
    const int nn = std::min(nbc, nb - b0);
    const int want = (b0 + nn >= nb) ? npatch - done
                                      : std::min(npatch - done, (int)((long long)npatch * (b0 + nn) / nb) - done);
    if (want <= 0) continue;
    const dim3 g2(64, nn);
    if (c.mixed) {
      RS_CUDA(cudaMemcpyAsync(X, w.psi.as<float>() + (size_t)b0 * vol, sizeof(float) * vol * nn,
                              cudaMemcpyDeviceToDevice, c.stream));
    } else {
      RS_TRY(convert_d2f(c, w.psi.as<double>() + (size_t)b0 * vol, X, vol * nn));
    }
    RS_TRY(hpsi_real<float>(c, k, s, X, HX, vol, nn));
    RS_CUDA(cudaMemsetAsync(d1, 0, sizeof(double) * 3 * nbc, c.stream));
    lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(X, X, d1, vol);
    lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(X, HX, d2, vol);
    lpc::k_grad_bands<<<g2, 256, 0, c.stream>>>(X, HX, G, d1, d2, vol);
    lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(G, G, d3, vol);
    lpc::k_scale<<<g2, 256, 0, c.stream>>>(G, G, d3, vol, 0);  // unit RMS
    c.launches += 5;
    // screened solve (T + sigma) Y = sigma G, Y0 = G
    RS_CUDA(cudaMemcpyAsync(Y, G, sizeof(float) * vol * nn, cudaMemcpyDeviceToDevice, c.stream));
    RS_TRY(kinetic_shifted(c, Y, HX, vol, nn, sigma));
    lpc::k_tcg_init<<<4 * 148, 256, 0, c.stream>>>(G, HX, R, P, (float)sigma, vol * nn);
    RS_CUDA(cudaMemsetAsync(d1, 0, sizeof(double) * nbc, c.stream));
    lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(R, R, d1, vol);
    c.launches += 2;
    for (int it = 0; it < iters; ++it) {
      RS_TRY(kinetic_shifted(c, P, HX, vol, nn, sigma));
      RS_CUDA(cudaMemsetAsync(d2, 0, sizeof(double) * 2 * nbc, c.stream));
      lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(P, HX, d2, vol);
      lpc::k_tcg_step<<<g2, 256, 0, c.stream>>>(Y, R, P, HX, d1, d2, vol);
      lpc::k_dot_bands<<<g2, 256, 0, c.stream>>>(R, R, d3, vol);
      lpc::k_tcg_dir<<<g2, 256, 0, c.stream>>>(P, R, d1, d3, vol);
      c.launches += 4;
      RS_CUDA(cudaMemcpyAsync(d1, d3, sizeof(double) * nbc, cudaMemcpyDeviceToDevice, c.stream));
    }
    // patch corners
    std::vector<int4> h(want);
    for (int i = 0; i < want; ++i) {
      h[i].x = (int)(rng() % (uint64_t)nn);
      h[i].y = (int)(rng() % (uint64_t)c.p.n1);
      h[i].z = (int)(rng() % (uint64_t)c.p.n2);
      h[i].w = (int)(rng() % (uint64_t)c.p.n3);
    }
    RS_CUDA(cudaMemcpyAsync(spec, h.data(), sizeof(int4) * want, cudaMemcpyHostToDevice, c.stream));
    lpc::k_extract<<<4 * 148, 256, 0, c.stream>>>(G, Y, spec, g_lpc.set_x.as<float>() + pv * g_lpc.set_n,
                                                  g_lpc.set_t.as<float>() + pv * g_lpc.set_n, want, pn, c.p.n1, c.p.n2,
                                                  c.p.n3);
    c.launches++;
    RS_CUDA(cudaStreamSynchronize(c.stream));  // h (host corners) must outlive the copy
    RS_TRY(check_launch("lpc_harvest"));
    g_lpc.set_n += want;
    done += want;
  }
  if (added) *added = done;
  return 0;
}

int lpc_dataset_size() { return g_lpc.set_n; }

// training on the harvested set
int lpc_train_set(Ctx& c, int margin, int epochs, int batch, double lr, uint64_t seed, double* losses) {
  RS_CHECK(g_lpc.set_n > 0, RSDFT_ERR_STATE, "training set is empty");
  return lpc_train(c, g_lpc.set_x.as<float>(), g_lpc.set_t.as<float>(), g_lpc.set_n, g_lpc.set_pn, margin, epochs,
                   batch, lr, seed, losses);
}

bool lpc_ready() { return g_lpc.ready; }

void lpc_release() {
  DBuf* bufs[] = {&g_lpc.w, &g_lpc.wb, &g_lpc.wt, &g_lpc.dw, &g_lpc.m, &g_lpc.v, &g_lpc.act, &g_lpc.dact,
                  &g_lpc.batch_x, &g_lpc.batch_t, &g_lpc.dy, &g_lpc.idx, &g_lpc.loss, &g_lpc.s2,
                  &g_lpc.set_x, &g_lpc.set_t, &g_lpc.hv, &g_lpc.hs, &g_lpc.io_a, &g_lpc.io_b,
                  &g_lpc.tcw, &g_lpc.tca};
  for (DBuf* b : bufs) b->release();
  g_lpc.ready = false;
  g_lpc.set_cap = g_lpc.set_n = g_lpc.set_pn = 0;
}

}  // namespace rsdft

// ---------------------------------------------------------------------------
// C ABI (declared in include/rsdft_b200.h)
// ---------------------------------------------------------------------------
using namespace rsdft;

#define LPC_CTX()                                                                      \
  Ctx* cp_ = ctx();                                                                    \
  RS_CHECK(cp_ != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");     \
  Ctx& c = *cp_

static int stage(DBuf& buf, const float* src, size_t n, int mem, const float** out) {
  RS_CHECK(mem == RSDFT_MEM_HOST || mem == RSDFT_MEM_DEVICE, RSDFT_ERR_ARG, "bad memory space %d", mem);
  if (mem == RSDFT_MEM_DEVICE) {
    *out = src;
    return 0;
  }
  RS_TRY(buf.ensure(sizeof(float) * n));
  RS_CUDA(cudaMemcpy(buf.p, src, sizeof(float) * n, cudaMemcpyHostToDevice));
  *out = buf.as<float>();
  return 0;
}

extern "C" {

int rsdft_gpu_lpc_init(unsigned long long seed) {
  LPC_CTX();
  return lpc_init_weights(c, seed);
}

int rsdft_gpu_lpc_set_weights(const float* w, int n) {
  LPC_CTX();
  RS_CHECK(w && n == lpc::WTOT, RSDFT_ERR_ARG, "weights: %d values given, the network has %d", n, lpc::WTOT);
  return lpc_set_weights(c, w);
}

int rsdft_gpu_lpc_get_weights(float* w, int n) {
  LPC_CTX();
  RS_CHECK(w && n == lpc::WTOT, RSDFT_ERR_ARG, "weights: room for %d values, the network has %d", n, lpc::WTOT);
  return lpc_get_weights(c, w);
}

int rsdft_gpu_lpc_forward(const float* x, float* y, int nb, int n1, int n2, int n3, int periodic, int mem) {
  LPC_CTX();
  RS_CHECK(x && y && nb > 0 && n1 > 0 && n2 > 0 && n3 > 0, RSDFT_ERR_ARG, "bad lpc_forward arguments");
  const size_t n = (size_t)nb * n1 * n2 * n3;
  const float* dx;
  RS_TRY(stage(g_lpc.io_a, x, n, mem, &dx));
  float* dy = y;
  if (mem == RSDFT_MEM_HOST) {
    RS_TRY(g_lpc.io_b.ensure(sizeof(float) * n));
    dy = g_lpc.io_b.as<float>();
  }
  RS_TRY(lpc_forward(c, dx, dy, nb, n1, n2, n3, periodic));
  if (mem == RSDFT_MEM_HOST) RS_CUDA(cudaMemcpyAsync(y, dy, sizeof(float) * n, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int rsdft_gpu_lpc_loss_grad(const float* x, const float* t, int nb, int n, int margin, double* loss, float* grad,
                            int mem) {
  LPC_CTX();
  RS_CHECK(x && t && nb > 0 && n > 0 && margin >= 0, RSDFT_ERR_ARG, "bad lpc_loss_grad arguments");
  const size_t cnt = (size_t)nb * n * n * n;
  const float *dx, *dt;
  RS_TRY(stage(g_lpc.io_a, x, cnt, mem, &dx));
  RS_TRY(stage(g_lpc.io_b, t, cnt, mem, &dt));
  return lpc_loss_grad(c, dx, dt, nb, n, margin, loss, grad);
}

int rsdft_gpu_lpc_dataset(int capacity, int patch) {
  LPC_CTX();
  return lpc_dataset(c, capacity, patch);
}

int rsdft_gpu_lpc_harvest(int k, int s, int npatch, double sigma, int iters, unsigned long long seed, int* added) {
  LPC_CTX();
  RS_CHECK(k >= 1 && k <= c.p.nk && s >= 1 && s <= c.p.nspin && npatch >= 0, RSDFT_ERR_ARG,
           "bad lpc_harvest arguments");
  return lpc_harvest(c, k - 1, s - 1, npatch, sigma, iters, seed, added);
}

int rsdft_gpu_lpc_dataset_get(int first, int count, float* x, float* t) {
  LPC_CTX();
  RS_CHECK(first >= 0 && count >= 0 && first + count <= g_lpc.set_n, RSDFT_ERR_ARG,
           "patches [%d, %d) outside the %d harvested", first, first + count, g_lpc.set_n);
  const size_t pv = (size_t)g_lpc.set_pn * g_lpc.set_pn * g_lpc.set_pn;
  if (x)
    RS_CUDA(cudaMemcpyAsync(x, g_lpc.set_x.as<float>() + pv * first, sizeof(float) * pv * count,
                            cudaMemcpyDeviceToHost, c.stream));
  if (t)
    RS_CUDA(cudaMemcpyAsync(t, g_lpc.set_t.as<float>() + pv * first, sizeof(float) * pv * count,
                            cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int rsdft_gpu_lpc_dataset_add(const float* x, const float* t, int count, int* added) {
  LPC_CTX();
  (void)c;
  RS_CHECK(x && t && count >= 0, RSDFT_ERR_ARG, "bad lpc_dataset_add arguments");
  RS_CHECK(g_lpc.set_cap > 0, RSDFT_ERR_STATE, "no training set: call lpc_dataset first");
  const int n = std::min(count, g_lpc.set_cap - g_lpc.set_n);
  const size_t pv = (size_t)g_lpc.set_pn * g_lpc.set_pn * g_lpc.set_pn;
  if (n > 0) {
    RS_CUDA(cudaMemcpy(g_lpc.set_x.as<float>() + pv * g_lpc.set_n, x, sizeof(float) * pv * n, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemcpy(g_lpc.set_t.as<float>() + pv * g_lpc.set_n, t, sizeof(float) * pv * n, cudaMemcpyHostToDevice));
    g_lpc.set_n += n;
  }
  if (added) *added = std::max(0, n);
  return 0;
}

int rsdft_gpu_lpc_train(int margin, int epochs, int batch, double lr, unsigned long long seed, double* losses) {
  LPC_CTX();
  return lpc_train_set(c, margin, epochs, batch, lr, seed, losses);
}

int rsdft_gpu_lpc_precond_f(const float* g, float* pg, int nb, int mem) {
  LPC_CTX();
  RS_CHECK(!c.cplx, RSDFT_ERR_UNSUPPORTED, "the learned preconditioner is built for the real Gamma build");
  RS_CHECK(g && pg && nb >= 0, RSDFT_ERR_ARG, "bad lpc_precond arguments");
  if (nb == 0) return 0;
  const size_t n = (size_t)nb * c.ng;
  const float* dg;
  RS_TRY(stage(g_lpc.io_a, g, n, mem, &dg));
  float* dp = pg;
  if (mem == RSDFT_MEM_HOST) {
    RS_TRY(g_lpc.io_b.ensure(sizeof(float) * n));
    dp = g_lpc.io_b.as<float>();
  }
  RS_TRY(lpc_apply(c, dg, dp, nb));
  if (mem == RSDFT_MEM_HOST) RS_CUDA(cudaMemcpyAsync(pg, dp, sizeof(float) * n, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int rsdft_gpu_lpc_inference(int mode) {
  LPC_CTX();
  RS_CHECK(mode == 0 || mode == 1, RSDFT_ERR_ARG, "inference mode %d: 0 (tensor cores) or 1 (FP32)", mode);
  c.lpc_fp32 = mode;
  return 0;
}

int rsdft_gpu_lpc_status(int* ready, int* pc_in_use, int* fallbacks, int* dataset) {
  LPC_CTX();
  if (ready) *ready = g_lpc.ready ? 1 : 0;
  if (pc_in_use) *pc_in_use = pc_effective(c);
  if (fallbacks) *fallbacks = c.lpc_fallbacks;
  if (dataset) *dataset = g_lpc.set_n;
  return 0;
}

}  // extern "C"
