// FP32 hpsi stencil for the real8 (Gamma) build on packed FP32 pairs.
//
// Same streaming design as the FP64 kernel (a CTA owns an N1 x TY column of one band, stages
// each xy-plane and its V_loc tile by bulk copies through an mbarrier ring, pushes z taps into
// 2*Md+1 rotating register accumulators, and takes the nonlocal scatter plane by plane from
// the nonlocal warps), with the arithmetic on float2 pairs of neighbouring x points through
// sm_100's packed FP32 instructions (__ffma2_rn / __fadd2_rn): y taps, z taps and the centre
// term act on aligned pairs directly; x taps pair the symmetric +-m neighbours and use the
// packed form for even m (aligned windows) and scalar FMAs for odd m.
// Reference semantics as in hpsi.cu: src/kinetic/d_kinetic_sol_module.f90:244-292 for the
// kinetic + V_loc part, src/ps_nloc_mr_module.f90:1159-1258 for the nonlocal part.
#include "stencil.cuh"

namespace rsdft {

namespace {

__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ float2 lo(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi(const float4& v) { return make_float2(v.z, v.w); }
__device__ __forceinline__ float2 dup(float c) { return make_float2(c, c); }

constexpr int R = 2;  // rows per thread
constexpr int P = 2;  // float2 pairs per row (4 x points)

// z push for rotation slot S: acc[S] += t, acc[S -+ m] += cz_m v, then emit slot S - Md
template <int MD, int S>
__device__ __forceinline__ void zpush(float2 (&acc)[2 * MD + 1][R][P], const float2 (&v)[R][P],
                                      const float2 (&t)[R][P], const float (&cz)[MD], bool fin, float* orow, int n1,
                                      const bool (&rowok)[R]) {
  constexpr int NQ = 2 * MD + 1;
  if constexpr (S < NQ) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) acc[S][r][j] = __fadd2_rn(acc[S][r][j], t[r][j]);
#pragma unroll
    for (int m = 1; m <= MD; ++m) {
      const float2 c = dup(cz[m - 1]);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) {
          acc[(S - m + NQ) % NQ][r][j] = __ffma2_rn(c, v[r][j], acc[(S - m + NQ) % NQ][r][j]);
          acc[(S + m) % NQ][r][j] = __ffma2_rn(c, v[r][j], acc[(S + m) % NQ][r][j]);
        }
    }
    constexpr int FS = (S + NQ - MD) % NQ;
    if (fin) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (rowok[r])
          *reinterpret_cast<float4*>(orow + (size_t)r * n1) =
              make_float4(acc[FS][r][0].x, acc[FS][r][0].y, acc[FS][r][1].x, acc[FS][r][1].y);
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) acc[FS][r][j] = make_float2(0.f, 0.f);
  }
}

#define RS_ZP_CASE(S_)                                           \
  case S_:                                                       \
    zpush<MD, S_>(acc, v, t, a.cz, fin, orow, n1, rowok);        \
    break;

}  // namespace

template <int MD, int S, int S2>
__global__ void __launch_bounds__(256, 1) k_stencil_f32(const StArgs<float, MD> a) {
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + 3) / 4;  // float4 chunks of x halo per side
  extern __shared__ __align__(128) unsigned char smem[];
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const StLayout L = smem_layout<float>(S, S2, a.stage_elems, a.vl_elems, a.nl_elems, a.ldc, a.rec_slots,
                                     a.rec_slot_bytes);
  float* stages = reinterpret_cast<float*>(smem);
  const int sstride = a.stage_elems + a.vl_elems;
  float* nlbuf = reinterpret_cast<float*>(smem + L.nlbuf);
  float* coef_s = reinterpret_cast<float*>(smem + L.coef);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* nlfull = bar + S;
  uint64_t* nlempty = nlfull + S2;
  uint64_t* recfull = nlempty + S2;
  int4* rechdr = reinterpret_cast<int4*>(smem + L.hdr);
  unsigned char* recbuf = smem + L.rec;

  const int tid = threadIdx.x;
  const int nthr_c = a.nthr_c;
  const bool active = tid < a.nact;
  const int tx = tid % a.bx, ty = tid / a.bx;
  const int x0 = tx * 4;
  const int yl = ty * R;
  const int y0 = blockIdx.x * a.tile_y;
  const int z0 = blockIdx.y * a.tz;
  const int zend = min(z0 + a.tz, n3);
  const int rows = a.tile_y + 2 * MD;
  const int nplanes = (zend - z0) + 2 * MD;
  const int ty_valid = min(a.tile_y, n2 - y0);
  const long long band = blockIdx.z;
  const float* src = a.psi + band * a.ld;
  float* dst = a.out + band * a.ld;
  const bool nl_on = a.rec_rowptr != nullptr;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
#pragma unroll
    for (int s = 0; s < S2; ++s) {
      mbar_init(&nlfull[s], kNLW);
      mbar_init(&nlempty[s], nthr_c);
    }
    for (int s = 0; s < a.rec_slots; ++s) mbar_init(&recfull[s], 1);
    fence_mbar_init();
  }
  if (nl_on)
    for (int i = tid; i < a.ldc; i += blockDim.x) coef_s[i] = a.coef[band * a.ldc + i];
  __syncthreads();

  if (tid >= nthr_c) {
    if (nl_on) nl_warps<float, MD, S2>(a, nlbuf, coef_s, nlfull, nlempty, recfull, rechdr, recbuf, tid, nthr_c, z0, zend, y0, ty_valid);
    return;
  }

  auto issue = [&](int q) {
    const int zg = pmod(z0 - MD + q, n3);
    float* st = stages + (size_t)(q % S) * sstride;
    uint64_t* br = &bar[q % S];
    const int p = z0 - MD + q;
    const bool inch = p >= z0 && p < zend;
    const uint32_t bytes = (uint32_t)((size_t)rows * n1 * 4) + (inch ? (uint32_t)((size_t)ty_valid * n1 * 4) : 0u);
    mbar_arrive_expect_tx(br, bytes);
    int r = 0;
    while (r < rows) {
      const int gy = pmod(y0 - MD + r, n2);
      const int len = min(rows - r, n2 - gy);
      bulk_g2s(st + (size_t)r * n1, src + ((size_t)zg * n2 + gy) * n1, (uint32_t)((size_t)len * n1 * 4), br);
      r += len;
    }
    if (inch) bulk_g2s(st + a.stage_elems, a.vloc + ((size_t)p * n2 + y0) * n1, (uint32_t)((size_t)ty_valid * n1 * 4), br);
  };
  if (tid == 0)
    for (int q = 0; q < S - 1 && q < nplanes; ++q) issue(q);

  bool rowok[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rowok[r] = active && (yl + r) < ty_valid;
  // x-window chunk offsets (wrapped once per thread)
  int xl[NCH], xr[NCH];
#pragma unroll
  for (int ch = 1; ch <= NCH; ++ch) {
    xl[ch - 1] = pmod(x0 - 4 * ch, n1);
    xr[ch - 1] = pmod(x0 + 4 * ch, n1);
  }
  const int yrow = active ? yl : 0;

  float2 acc[NQ][R][P];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) acc[q][r][j] = make_float2(0.f, 0.f);

  int issued_upto = min(S - 1, nplanes);
  bool aborted = false;
  for (int q = 0; q < nplanes; ++q) {
    if (tid == 0 && q + S - 1 < nplanes) {
      fence_proxy_async_smem();
      issue(q + S - 1);
      issued_upto = q + S;
    }
    bool ok = mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
    const float* pl = stages + (size_t)(q % S) * sstride;
    const float* prow = pl + (size_t)(yrow + MD) * n1;  // own first row
    const int p = z0 - MD + q;
    const bool inch = p >= z0 && p < zend;
    float2 v[R][P], t[R][P];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float4 c = lds4(prow + (size_t)r * n1 + x0);
      v[r][0] = lo(c);
      v[r][1] = hi(c);
#pragma unroll
      for (int j = 0; j < P; ++j) t[r][j] = make_float2(0.f, 0.f);
    }
    if (inch) {
      const int pi = p - z0;
      const int slot = pi % S2;
      const float* nl = nlbuf + (size_t)slot * a.nl_elems;
      if (nl_on) ok = mbar_wait_bounded(&nlfull[slot], (uint32_t)((pi / S2) & 1), kWaitPolls) && ok;
      // centre: (c0 + V_loc) psi + nonlocal
      const float2 c0 = dup(a.c0);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float4 vl = lds4(pl + a.stage_elems + (size_t)(yrow + r) * n1 + x0);
        float4 nv = make_float4(0.f, 0.f, 0.f, 0.f);
        if (nl_on) nv = lds4(nl + (size_t)(yrow + r) * n1 + x0);
        t[r][0] = __ffma2_rn(__fadd2_rn(c0, lo(vl)), v[r][0], lo(nv));
        t[r][1] = __ffma2_rn(__fadd2_rn(c0, hi(vl)), v[r][1], hi(nv));
      }
      // x taps: window w[-4 NCH .. 4 NCH + 3] of the staged (periodic) row
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float* row = prow + (size_t)r * n1;
        float w[(2 * NCH + 1) * 4];
        w[4 * NCH + 0] = v[r][0].x;
        w[4 * NCH + 1] = v[r][0].y;
        w[4 * NCH + 2] = v[r][1].x;
        w[4 * NCH + 3] = v[r][1].y;
#pragma unroll
        for (int ch = 1; ch <= NCH; ++ch) {
          const float4 l = lds4(row + xl[ch - 1]);
          const float4 rr = lds4(row + xr[ch - 1]);
          w[4 * (NCH - ch) + 0] = l.x;
          w[4 * (NCH - ch) + 1] = l.y;
          w[4 * (NCH - ch) + 2] = l.z;
          w[4 * (NCH - ch) + 3] = l.w;
          w[4 * (NCH + ch) + 0] = rr.x;
          w[4 * (NCH + ch) + 1] = rr.y;
          w[4 * (NCH + ch) + 2] = rr.z;
          w[4 * (NCH + ch) + 3] = rr.w;
        }
        constexpr int C = 4 * NCH;  // index of x0 in w
#pragma unroll
        for (int m = 1; m <= MD; ++m) {
          const float cm = a.cx[m - 1];
          if ((m & 1) == 0) {
#pragma unroll
            for (int j = 0; j < P; ++j) {
              const float2 lp = make_float2(w[C + 2 * j - m], w[C + 2 * j + 1 - m]);
              const float2 rp = make_float2(w[C + 2 * j + m], w[C + 2 * j + 1 + m]);
              t[r][j] = __ffma2_rn(dup(cm), __fadd2_rn(lp, rp), t[r][j]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < P; ++j) {
              t[r][j].x = fmaf(cm, w[C + 2 * j - m] + w[C + 2 * j + m], t[r][j].x);
              t[r][j].y = fmaf(cm, w[C + 2 * j + 1 - m] + w[C + 2 * j + 1 + m], t[r][j].y);
            }
          }
        }
      }
      // y taps: rows yl-MD .. yl+R-1+MD of the stage; the own rows come from v
#pragma unroll
      for (int dy = -MD; dy < R + MD; ++dy) {
        float2 rv[P];
        if (dy >= 0 && dy < R) {
#pragma unroll
          for (int j = 0; j < P; ++j) rv[j] = v[(dy >= 0 && dy < R) ? dy : 0][j];
        } else {
          const float4 c = lds4(prow + (ptrdiff_t)dy * n1 + x0);
          rv[0] = lo(c);
          rv[1] = hi(c);
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int m = dy > r ? dy - r : r - dy;
          if (m >= 1 && m <= MD) {
            const float2 cm = dup(a.cy[(m >= 1 && m <= MD ? m : 1) - 1]);
#pragma unroll
            for (int j = 0; j < P; ++j) t[r][j] = __ffma2_rn(cm, rv[j], t[r][j]);
          }
        }
      }
      if (nl_on) mbar_arrive(&nlempty[slot]);
    }
    const int zo = p - MD;
    const bool fin = zo >= z0 && zo < zend;
    float* orow = dst + ((size_t)(fin ? zo : 0) * n2 + (y0 + yl)) * n1 + x0;
    switch (q % NQ) {
      RS_ZP_CASE(0) RS_ZP_CASE(1) RS_ZP_CASE(2) RS_ZP_CASE(3) RS_ZP_CASE(4) RS_ZP_CASE(5)
      RS_ZP_CASE(6) RS_ZP_CASE(7) RS_ZP_CASE(8) RS_ZP_CASE(9) RS_ZP_CASE(10) RS_ZP_CASE(11)
      RS_ZP_CASE(12)
      default: break;
    }
    if (bar_or(!ok, nthr_c)) {
      aborted = true;
      if (tid == 0) atomicOr(a.status, DEV_WAIT_TIMEOUT);
      break;
    }
  }
  if (aborted && tid == 0) {
    // drain copies still in flight before the CTA's shared memory is released
    for (int q = 0; q < issued_upto; ++q) mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
  }
}

template <int MD, int S, int S2>
int launch_stencil_f32(const StArgs<float, MD>& a, dim3 grid, dim3 block, size_t smem, cudaStream_t st) {
  auto kern = k_stencil_f32<MD, S, S2>;
  static bool attr_done = false;  // one per template instantiation
  if (!attr_done) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 225 * 1024));
    attr_done = true;
  }
  kern<<<grid, block, smem, st>>>(a);
  return 0;
}

template <int MD, int S, int S2>
int stencil_f32_block_limit(int* max_threads) {
  cudaFuncAttributes fa{};
  RS_CUDA(cudaFuncGetAttributes(&fa, k_stencil_f32<MD, S, S2>));
  *max_threads = fa.maxThreadsPerBlock;
  return 0;
}

template int stencil_f32_block_limit<6, 6, 3>(int*);
template int stencil_f32_block_limit<4, 6, 3>(int*);
template int launch_stencil_f32<6, 6, 3>(const StArgs<float, 6>&, dim3, dim3, size_t, cudaStream_t);
template int launch_stencil_f32<4, 6, 3>(const StArgs<float, 4>&, dim3, dim3, size_t, cudaStream_t);

}  // namespace rsdft
