// Fused, z-streamed precond_hprsdft for FP32 bands plus the CG direction update.
//
// Reference: precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270; 7-point
// operator precond_cg_mat2_omp, :288-361), the dot <Pg|g> and the direction update
// p = Pg + (rb / gkgk) p of the CG step (src/conjugate_gradient/cg_module.f90:254-283).
//
// The mloop CG steps of the preconditioner are evaluated in the s-step form of cg.cu: with
// A = c0 (B + I) and r0 = G - A G, every vector of that CG lies in span{v_i = B^i r0, i < m}, so
// PG = G + sum_i xi_i v_i where xi comes from a small recurrence on the moments
// mu_j = <r0 | B^j r0>, j < 2m.  Here the whole chain G -> r0 -> v_1 -> ... is computed on the
// fly, plane by plane, inside one kernel, and the bands are touched twice instead of 3m + 3
// times (plus the 3 passes of the direction update):
//
//   moments pass  reads G once; accumulates mu_0 .. mu_{2m-1}, nu_i = <G | v_i> and <G | G>.
//   (scalars)     per band: xi from the recurrence, <PG|G> = <G|G> + sum_i xi_i nu_i (exact in
//                 exact arithmetic, so PG itself is never stored), rb, beta = rb / gkgk.
//   update pass   reads G once more and p; recomputes r0 .. v_{m-1}, forms
//                 PG = G + sum xi_i v_i and writes p = PG + beta p (p = PG on the first step).
//
// Design (B200, sm_100a): persistent CTAs (one per SM) walk items (band, y-tile); an item streams
// all z planes of its column of full x-rows.  A G plane of the tile (tile rows plus a periodic
// halo of one row per chain level, split into at most a few contiguous segments) arrives by bulk
// copy (TMA engine, cp.async.bulk + mbarrier) into a ring of slots a few planes ahead.  Level j of
// the chain keeps its last planes in a shared-memory ring (rows shrink by one per side per
// level); at step t level j computes plane t - 1 - 2 j from level j - 1's planes t - 2 - 2 j ..
// t - 2 j, all written in earlier steps, so the levels of a step are independent work units
// (32 consecutive 4-real groups of one level's plane tile, one per warp) behind one CTA barrier
// per step.  Every lane owns 4 consecutive reals (16-byte shared loads at 32-bit shared
// addresses, packed FP32x2 arithmetic); the x neighbours come by warp shuffle when a row is 16
// or 32 groups wide, else from shared memory.
// Moments accumulate per thread in packed FP32 pairs, across threads in FP64.  All waits are
// bounded: a thread that gives up sets the device status word; the CTA then waits (bounded) for
// its own copies in flight and leaves.
#include "cgk.cuh"
#include "ptx.cuh"
#include "stencil.cuh"

namespace rsdft {

namespace {

constexpr int kPzMaxThreads = 1024;
constexpr int kPzMaxWarps = kPzMaxThreads / 32;
constexpr int kPzGSlots = 8;  // G ring slots (a power of two): planes t - KG .. t + 8 - KG - 1

struct PzArgs {
  const float* G;     // gradients, [nbb][ng] reals
  float* P;           // CG directions (update pass: in place)
  double* part;       // moments pass: partials [nbb][ytiles][kPS]
  const double* sc;   // per-band scalars [S_COUNT][nbb]
  int nbb;
  int L, n2, n3;      // reals per x-row (n1 * components), rows, planes
  int ty, ytiles;     // tile rows, tiles per plane
  int nslot;          // G ring slots
  size_t ng;          // reals per band
  float a0, a1, a2, a3;  // A = a0 I + a_d (shift_+d + shift_-d)
  float b1, b2, b3;      // B = (A - a0 I) / a0
  int first;             // first CG step: p = PG
  int threads;           // CTA size
  unsigned* status;
  uint32_t polls;
};

__device__ __forceinline__ double pz_sc(const PzArgs& a, int which, int b) { return a.sc[(size_t)which * a.nbb + b]; }

// 16-byte (and smaller) shared-memory accesses at 32-bit shared addresses
__device__ __forceinline__ float4 sld4(uint32_t a) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ void sst4(uint32_t a, const float4& v) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
               : "memory");
}
__device__ __forceinline__ float sld1(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float2 sld2(uint32_t a) {
  float2 v;
  asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
  return v;
}

// a group of 4 reals as two packed pairs
struct Q4 {
  float2 lo, hi;
};
__device__ __forceinline__ Q4 q4(const float4& v) { return {make_float2(v.x, v.y), make_float2(v.z, v.w)}; }
__device__ __forceinline__ float4 f4(const Q4& q) { return make_float4(q.lo.x, q.lo.y, q.hi.x, q.hi.y); }
__device__ __forceinline__ Q4 qadd(const Q4& a, const Q4& b) { return {__fadd2_rn(a.lo, b.lo), __fadd2_rn(a.hi, b.hi)}; }
__device__ __forceinline__ Q4 qfma(float2 c, const Q4& a, const Q4& b) {
  return {__ffma2_rn(c, a.lo, b.lo), __ffma2_rn(c, a.hi, b.hi)};
}
__device__ __forceinline__ Q4 qmul(float2 c, const Q4& a) { return {__fmul2_rn(c, a.lo), __fmul2_rn(c, a.hi)}; }
// <x|y> of a group accumulated into a packed FP32 pair (the pass adds the pairs of all threads
// in FP64 at the end of each item, as the multi-pass kernels add their per-thread FP32 sums)
__device__ __forceinline__ void qdot(float2& acc, const Q4& x, const Q4& y) {
  acc = __ffma2_rn(x.hi, y.hi, __ffma2_rn(x.lo, y.lo, acc));
}

// x neighbours (x - 1, x + 1 in component units) of the group c at group g of a staged row
// (row address rowa); NGS > 0: a row is NGS consecutive lanes, neighbours by shuffle
template <int NCP, int NGS>
__device__ __forceinline__ void pz_xnb(uint32_t rowa, int g, int L, const float4& c, Q4& xm, Q4& xp) {
  float l0 = 0.f, l1, r0, r1 = 0.f;
  if constexpr (NGS > 0) {
    const int gl = (g - 1) & (NGS - 1), gr = (g + 1) & (NGS - 1);
    l1 = __shfl_sync(0xffffffffu, c.w, gl, NGS);
    r0 = __shfl_sync(0xffffffffu, c.x, gr, NGS);
    if constexpr (NCP == 2) {
      l0 = __shfl_sync(0xffffffffu, c.z, gl, NGS);
      r1 = __shfl_sync(0xffffffffu, c.y, gr, NGS);
    }
  } else {
    const int xl = (g == 0 ? L : 4 * g) - NCP;
    const int xr = 4 * g + 4 == L ? 0 : 4 * g + 4;
    if constexpr (NCP == 1) {
      l1 = sld1(rowa + 4u * (uint32_t)xl);
      r0 = sld1(rowa + 4u * (uint32_t)xr);
    } else {
      const float2 lp = sld2(rowa + 4u * (uint32_t)xl), rp = sld2(rowa + 4u * (uint32_t)xr);
      l0 = lp.x;
      l1 = lp.y;
      r0 = rp.x;
      r1 = rp.y;
    }
  }
  if constexpr (NCP == 1) {
    xm = {make_float2(l1, c.x), make_float2(c.y, c.z)};
    xp = {make_float2(c.y, c.z), make_float2(c.w, r0)};
  } else {
    xm = {make_float2(l0, l1), make_float2(c.x, c.y)};
    xp = {make_float2(c.z, c.w), make_float2(r0, r1)};
  }
}

// Bounded wait on a G slot that also leaves when another thread of the CTA gave up.
__device__ __forceinline__ bool pz_wait(uint64_t* bar, uint32_t parity, const volatile int* abort_flag,
                                        uint32_t polls) {
  for (uint32_t it = 0; it < polls; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 63u) {
      if (*abort_flag) return false;
      __nanosleep(64);
    }
  }
  return false;
}

// Shared-memory layout of one CTA (byte addresses): the G ring, then one ring per stored level.
template <int NLEV>
struct PzLayout {
  uint32_t gbase, gps;         // G ring base, bytes per slot
  uint32_t lbase[NLEV], lps[NLEV];
  int lrd[NLEV];               // planes per level ring
  uint32_t rb;                 // bytes per staged row
};

// ring depth of stored level j: 4 planes (the one written this step and the three its
// successor reads); the update pass keeps level j for its combine step 2 (M - 1 - j) planes later
template <int M, bool MOM>
__host__ __device__ constexpr int pz_depth(int j) {
  return MOM ? 4 : (2 * M - 1 - 2 * j > 4 ? 8 : 4);
}

// One work unit of a step: 32 consecutive (row, group) items of chain level J on its plane r.
template <int M, int NCP, int NGS, bool MOM, int J>
__device__ __forceinline__ void pz_task(const PzArgs& a, const PzLayout<(MOM ? M + 1 : M)>& ly, int unit, int r,
                                        uint32_t gslot_r, uint32_t gslot_m, uint32_t gslot_p, int tyv, int y0,
                                        float* Pb, float2 (&acc)[(MOM ? 3 * M + 1 : 1)], const float2 (&xi)[M],
                                        float2 beta2, int lane) {
  constexpr int NLEV = MOM ? M + 1 : M;
  constexpr int NST = NLEV - 1;
  constexpr int H = NLEV - 1 - J;  // halo rows of level J on each side
  const int L = a.L, NGR = L >> 2;
  const int rows = a.ty + 2 * H;
  const int total = rows * NGR;
  const int idx0 = unit * 32 + lane;
  const bool act = idx0 < total;
  const int idx = act ? idx0 : total - 1;
  int rho, g;
  if constexpr (NGS > 0) {
    rho = idx / NGS;
    g = idx & (NGS - 1);
  } else {
    rho = idx / NGR;
    g = idx - rho * NGR;
  }
  const uint32_t rb = ly.rb;
  const uint32_t lo = 16u * (uint32_t)g;
  uint32_t sm, s0, sp;  // source planes z - 1, z, z + 1
  if constexpr (J == 0) {
    sm = ly.gbase + gslot_m * ly.gps;
    s0 = ly.gbase + gslot_r * ly.gps;
    sp = ly.gbase + gslot_p * ly.gps;
  } else {
    constexpr int RM = pz_depth<M, MOM>(J - 1) - 1;
    const uint32_t ps = ly.lps[J - 1], b0 = ly.lbase[J - 1];
    sm = b0 + (uint32_t)((r - 1) & RM) * ps;
    s0 = b0 + (uint32_t)(r & RM) * ps;
    sp = b0 + (uint32_t)((r + 1) & RM) * ps;
  }
  const uint32_t ro = (uint32_t)(rho + 1) * rb + lo;
  const float4 c4 = sld4(s0 + ro);
  const Q4 c = q4(c4);
  const Q4 ys = qadd(q4(sld4(s0 + ro - rb)), q4(sld4(s0 + ro + rb)));
  const Q4 zs = qadd(q4(sld4(sm + ro)), q4(sld4(sp + ro)));
  Q4 xm, xp;
  pz_xnb<NCP, NGS>(s0 + (uint32_t)(rho + 1) * rb, g, L, c4, xm, xp);
  const Q4 xs = qadd(xm, xp);
  Q4 out;
  if constexpr (J == 0) {
    // r0 = c - A c, A c = a0 c + a1 (x- + x+) + a2 (y- + y+) + a3 (z- + z+)
    Q4 ag = qmul(make_float2(a.a0, a.a0), c);
    ag = qfma(make_float2(a.a1, a.a1), xs, ag);
    ag = qfma(make_float2(a.a2, a.a2), ys, ag);
    ag = qfma(make_float2(a.a3, a.a3), zs, ag);
    out = {__fadd2_rn(c.lo, make_float2(-ag.lo.x, -ag.lo.y)), __fadd2_rn(c.hi, make_float2(-ag.hi.x, -ag.hi.y))};
  } else {
    out = qmul(make_float2(a.b1, a.b1), xs);
    out = qfma(make_float2(a.b2, a.b2), ys, out);
    out = qfma(make_float2(a.b3, a.b3), zs, out);
  }
  if (!act) return;
  if constexpr (J < NST)
    sst4(ly.lbase[J] + (uint32_t)(r & (pz_depth<M, MOM>(J) - 1)) * ly.lps[J] + (uint32_t)rho * rb + lo, f4(out));
  const int yo = rho - H;
  if (r < NLEV || r >= NLEV + a.n3 || yo < 0 || yo >= tyv) return;
  if constexpr (MOM) {
    if constexpr (J == 0) {
      qdot(acc[0], out, out);
      qdot(acc[2 * M], c, out);
      qdot(acc[3 * M], c, c);
    } else if constexpr (J < M) {
      const Q4 gv = q4(sld4(ly.gbase + gslot_r * ly.gps + (uint32_t)(rho + J + 1) * rb + lo));
      qdot(acc[2 * J - 1], c, out);
      qdot(acc[2 * J], out, out);
      qdot(acc[2 * M + J], gv, out);
    } else {
      qdot(acc[2 * M - 1], c, out);
    }
  } else if constexpr (J == NLEV - 1) {
    // PG = G + sum_i xi_i v_i at an own point (this level has no halo rows), p = PG + beta p
    Q4 pg = q4(sld4(ly.gbase + gslot_r * ly.gps + (uint32_t)(rho + NLEV) * rb + lo));
#pragma unroll
    for (int i = 0; i < M - 1; ++i) {
      const int rmask = pz_depth<M, MOM>(i) - 1;
      const Q4 vi = q4(sld4(ly.lbase[i] + (uint32_t)(r & rmask) * ly.lps[i] + (uint32_t)(rho + (NLEV - 1 - i)) * rb + lo));
      pg = qfma(xi[i], vi, pg);
    }
    pg = qfma(xi[M - 1], out, pg);
    float4* pp = reinterpret_cast<float4*>(Pb + ((size_t)(r - NLEV) * a.n2 + (y0 + yo)) * L + 4 * g);
    if (!a.first) pg = qfma(beta2, q4(*pp), pg);
    *pp = f4(pg);
  }
}

// MOM: the moments pass (chain levels r0, v_1 .. v_{M-1}, B v_{M-1}); else the update pass
// (levels r0 .. v_{M-1}, then PG and p).  Level j works on plane t - 1 - 2 j at step t, so every
// level of a step reads only planes of earlier steps and one CTA barrier per step suffices.
template <int M, int NCP, int NGS, bool MOM>
__global__ void __launch_bounds__(kPzMaxThreads, 1) k_pcz(PzArgs a) {
  constexpr int NLEV = MOM ? M + 1 : M;   // chain levels computed
  constexpr int NST = NLEV - 1;           // levels kept in shared-memory rings
  constexpr int KG = 2 * M - 1 > 2 ? 2 * M - 1 : 2;  // oldest G plane read at step t: t - KG
  constexpr int NV = MOM ? 3 * M + 1 : 1;  // sums: mu_0..mu_{2M-1}, nu_0..nu_{M-1}, <G|G>
  extern __shared__ __align__(128) unsigned char pz_smem[];
  __shared__ double red[kPzMaxWarps][NV];
  const int L = a.L, NGR = L >> 2;
  const int rowsG = a.ty + 2 * NLEV;
  PzLayout<NLEV> ly;
  ly.rb = 4u * (uint32_t)L;
  ly.gbase = smem_u32(pz_smem);
  ly.gps = (uint32_t)rowsG * ly.rb;
  uint32_t off = (uint32_t)kPzGSlots * ly.gps;
#pragma unroll
  for (int j = 0; j < NLEV; ++j) {
    ly.lrd[j] = pz_depth<M, MOM>(j);
    ly.lps[j] = (uint32_t)(a.ty + 2 * (NLEV - 1 - j)) * ly.rb;
    ly.lbase[j] = ly.gbase + off;
    if (j < NST) off += (uint32_t)ly.lrd[j] * ly.lps[j];
  }
  uint64_t* full = reinterpret_cast<uint64_t*>(pz_smem + off);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(full + kPzGSlots);
  float* gring = reinterpret_cast<float*>(pz_smem);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPzGSlots; ++s) mbar_init(&full[s], 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  // work units (32 items) per level and step
  int ucum[NLEV + 1];
  ucum[0] = 0;
#pragma unroll
  for (int j = 0; j < NLEV; ++j) ucum[j + 1] = ucum[j] + ((a.ty + 2 * (NLEV - 1 - j)) * NGR + 31) / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int T = a.n3 + 3 * NLEV - 1;  // G planes streamed per item
  constexpr int D = kPzGSlots - KG - 1;  // planes requested ahead
  constexpr uint32_t GM = kPzGSlots - 1;
  uint32_t gseq = 0;  // G planes of earlier items of this CTA
  const int nitems = a.nbb * a.ytiles;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int b = item / a.ytiles, yt = item - b * a.ytiles;
    if (pz_sc(a, S_ACT, b) == 0.0) continue;
    const int y0 = yt * a.ty, tyv = min(a.ty, a.n2 - y0);
    const float* Gb = a.G + (size_t)b * a.ng;
    float* Pb = a.P + (size_t)b * a.ng;
    auto issue = [&](int r) {  // G plane r of the item (z = r - NLEV), rows y0 - NLEV ..
      const uint32_t q = gseq + (uint32_t)r;
      const int slot = (int)(q & GM);
      float* dst = gring + (size_t)slot * (ly.gps / 4);
      const int z = pmod(r - NLEV, a.n3);
      int y = pmod(y0 - NLEV, a.n2), left = rowsG;
      mbar_arrive_expect_tx(&full[slot], (uint32_t)rowsG * ly.rb);
      while (left > 0) {
        const int seg = min(left, a.n2 - y);
        bulk_g2s(dst, Gb + ((size_t)z * a.n2 + y) * L, (uint32_t)seg * ly.rb, &full[slot]);
        dst += (size_t)seg * L;
        left -= seg;
        y = 0;
      }
    };
    if (threadIdx.x == 0)
      for (int r = 0; r <= D && r < T; ++r) issue(r);
    float2 acc[NV];
#pragma unroll
    for (int d = 0; d < NV; ++d) acc[d] = make_float2(0.f, 0.f);
    float2 xi[M];
    float2 beta2 = make_float2(0.f, 0.f);
    if constexpr (!MOM) {
      const bool on = pz_sc(a, S_PCACT, b) != 0.0;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        const float x = on ? (float)pz_sc(a, S_XI0 + i, b) : 0.f;
        xi[i] = make_float2(x, x);
      }
      const float be = a.first ? 0.f : (float)pz_sc(a, S_BETA, b);
      beta2 = make_float2(be, be);
    } else {
#pragma unroll
      for (int i = 0; i < M; ++i) xi[i] = make_float2(0.f, 0.f);
    }
    for (int t = 0; t < T; ++t) {
      const uint32_t q = gseq + (uint32_t)t;
      const bool ok = pz_wait(&full[q & GM], (q / kPzGSlots) & 1u, abort_flag, a.polls);
      if (!ok) *abort_flag = 1;
      if (__syncthreads_or(!ok)) {
        if (threadIdx.x == 0) {
          atomicOr(a.status, DEV_WAIT_TIMEOUT);
          // wait for this CTA's copies still in flight before leaving
          const int last = min(T - 1, t + D);
          for (int r = t; r <= last; ++r) {
            const uint32_t qq = gseq + (uint32_t)r;
            mbar_wait_bounded(&full[qq & GM], (qq / kPzGSlots) & 1u, a.polls);
          }
        }
        return;
      }
      // levels whose inputs exist: level j starts at step 3 j + 2
      int jmax = -1;
#pragma unroll
      for (int j = 0; j < NLEV; ++j)
        if (t >= 3 * j + 2) jmax = j;
      int nunits = 0;
#pragma unroll
      for (int j = 0; j < NLEV; ++j)
        if (j == jmax) nunits = ucum[j + 1];
      for (int u = warp; u < nunits; u += nwarp) {
        int j = 0, ubase = 0;
#pragma unroll
        for (int jj = 1; jj < NLEV; ++jj)
          if (u >= ucum[jj]) {
            j = jj;
            ubase = ucum[jj];
          }
        const int r = t - 1 - 2 * j;
        const int unit = u - ubase;
        // G slots of planes r, r - 1, r + 1 (level 0 reads all three; later levels read plane r)
        const uint32_t gr = (gseq + (uint32_t)r) & GM;
        const uint32_t gm = (gr - 1) & GM, gp = (gr + 1) & GM;
        switch (j) {
          case 0: pz_task<M, NCP, NGS, MOM, 0>(a, ly, unit, r, gr, gm, gp, tyv, y0, Pb, acc, xi, beta2, lane); break;
          case 1: if constexpr (NLEV > 1) pz_task<M, NCP, NGS, MOM, (NLEV > 1 ? 1 : 0)>(a, ly, unit, r, gr, gm, gp, tyv, y0, Pb, acc, xi, beta2, lane); break;
          case 2: if constexpr (NLEV > 2) pz_task<M, NCP, NGS, MOM, (NLEV > 2 ? 2 : 0)>(a, ly, unit, r, gr, gm, gp, tyv, y0, Pb, acc, xi, beta2, lane); break;
          default: if constexpr (NLEV > 3) pz_task<M, NCP, NGS, MOM, (NLEV > 3 ? 3 : 0)>(a, ly, unit, r, gr, gm, gp, tyv, y0, Pb, acc, xi, beta2, lane); break;
        }
      }
      __syncthreads();
      // every read of this step is done: the slot of plane t - KG takes plane t + D + 1
      if (threadIdx.x == 0 && t + D + 1 < T) issue(t + D + 1);
    }
    gseq += (uint32_t)T;
    if constexpr (MOM) {
#pragma unroll
      for (int d = 0; d < NV; ++d) {
        double x = (double)acc[d].x + (double)acc[d].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][d] = x;
      }
      __syncthreads();
      if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < nwarp; ++w) s += red[w][threadIdx.x];
        a.part[((size_t)b * a.ytiles + yt) * kPS + threadIdx.x] = s;
      }
      __syncthreads();
    }
  }
}

// After the moments pass: xi, <PG|G>, rb, beta and gkgk per band (k_sc_beta's bookkeeping).
template <int M>
__global__ void k_pcz_sc(Blk kz, double c0, double dV, int first) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= kz.nbb) return;
  if (SC(kz, S_ACT, b) == 0.0) {
    SC(kz, S_PCACT, b) = 0.0;
    return;
  }
  double mu[8], xi[5];
  for (int j = 0; j < 2 * M; ++j) mu[j] = sum_part(kz, b, j);
  SC(kz, S_RR1, b) = mu[0];
  const bool on = !(mu[0] < 1.0e-24);  // cgpc_hprsdft_module.f90:181
  SC(kz, S_PCACT, b) = on ? 1.0 : 0.0;
  double pgg = sum_part(kz, b, 3 * M);
  if (on) {
    pcs_recurrence(mu, M, c0, xi);
    for (int i = 0; i < M; ++i) {
      SC(kz, S_XI0 + i, b) = xi[i];
      pgg += xi[i] * sum_part(kz, b, 2 * M + i);
    }
  }
  const double rb = pgg * dV;
  SC(kz, S_RB, b) = rb;
  SC(kz, S_BETA, b) = first ? 0.0 : rb / SC(kz, S_GKGK, b);
  SC(kz, S_GKGK, b) = rb;
}

struct PzPlan {
  int ty, ytiles, nslot, thr_mom, thr_upd;
  size_t smem_mom, smem_upd;
};

size_t pz_smem_bytes(int M, bool mom, int ty, int L, int nslot) {
  const int nlev = mom ? M + 1 : M;
  size_t rows = (size_t)nslot * (ty + 2 * nlev);
  for (int j = 0; j < nlev - 1; ++j) {
    const int rd = mom ? 4 : (2 * M - 1 - 2 * j > 4 ? 8 : 4);
    rows += (size_t)rd * (ty + 2 * (nlev - 1 - j));
  }
  return rows * 4 * (size_t)L + 8 * (size_t)nslot + 16;
}

// warps of a pass: the work units (32 items of a level plane tile) of one step, spread over the
// fewest rounds of at most 32 warps
int pz_threads(int M, bool mom, int ty, int ngr) {
  const int nlev = mom ? M + 1 : M;
  int units = 0;
  for (int j = 0; j < nlev; ++j) units += ((ty + 2 * (nlev - 1 - j)) * ngr + 31) / 32;
  const int rounds = (units + kPzMaxWarps - 1) / kPzMaxWarps;
  const int warps = (units + rounds - 1) / rounds;
  return std::max(4, warps) * 32;
}

constexpr size_t kPzSmemMax = 227 * 1024 - 4096;  // dynamic shared memory (static: the reduction scratch)

// Tile rows: the candidate that fits shared memory with the least computed rows per own row
// (halo rows of every level and the ragged last tile).
bool pz_plan(const Ctx& c, PzPlan& pl) {
  const int M = c.p.mloop;
  const int L = c.p.n1 * (c.cplx ? 2 : 1);
  const int ngr = L / 4;
  pl.nslot = kPzGSlots;
  double best = 1e30;
  bool found = false;
  for (int ty = std::min(32, c.p.n2); ty >= 1; --ty) {
    const size_t sm = pz_smem_bytes(M, true, ty, L, pl.nslot);
    if (sm > kPzSmemMax) continue;
    const int yt = (c.p.n2 + ty - 1) / ty;
    double rows = 0.0;
    for (int j = 0; j <= M; ++j) rows += ty + 2 * (M - j);
    const double cost = (double)yt * rows;
    if (cost < best - 1e-9) {
      best = cost;
      found = true;
      pl.ty = ty;
      pl.ytiles = yt;
      pl.smem_mom = sm;
      pl.smem_upd = pz_smem_bytes(M, false, ty, L, pl.nslot);
      pl.thr_mom = pz_threads(M, true, ty, ngr);
      pl.thr_upd = pz_threads(M, false, ty, ngr);
    }
  }
  return found;
}

template <int M, int NCP, int NGS, bool MOM>
int pz_launch(Ctx& c, PzArgs a, size_t smem, int grid) {
  auto kern = k_pcz<M, NCP, NGS, MOM>;
  static bool attr = false;  // one per instantiation
  if (!attr) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPzSmemMax));
    attr = true;
  }
  kern<<<grid, a.threads, smem, c.stream>>>(a);
  c.launches++;
  return 0;
}

template <int M, bool MOM>
int pz_dispatch(Ctx& c, PzArgs a, size_t smem, int grid, int ncp, int ngs, int threads) {
  a.threads = threads;
  if (ncp == 1) {
    if (ngs == 32) return pz_launch<M, 1, 32, MOM>(c, a, smem, grid);
    if (ngs == 16) return pz_launch<M, 1, 16, MOM>(c, a, smem, grid);
    return pz_launch<M, 1, 0, MOM>(c, a, smem, grid);
  }
  if (ngs == 32) return pz_launch<M, 2, 32, MOM>(c, a, smem, grid);
  if (ngs == 16) return pz_launch<M, 2, 16, MOM>(c, a, smem, grid);
  return pz_launch<M, 2, 0, MOM>(c, a, smem, grid);
}

}  // namespace

bool pc_fused_applies(const Ctx& c) {
  if (!c.mixed || c.pc_sstep != 2 || c.cggs) return false;
  if (c.p.mloop < 1 || c.p.mloop > 3) return false;
  const int L = c.p.n1 * (c.cplx ? 2 : 1);
  if (L % 4 != 0) return false;
  PzPlan pl;
  return pz_plan(c, pl);
}

size_t pc_fused_part_doubles(const Ctx& c, int nbb) {
  PzPlan pl;
  if (!pz_plan(c, pl)) return 0;
  return (size_t)kPS * (size_t)nbb * (size_t)pl.ytiles;
}

int pc_fused_step(Ctx& c, Blk& k, const float* G, float* P, int first) {
  RS_CHECK(pc_fused_applies(c), RSDFT_ERR_UNSUPPORTED, "fused preconditioner does not apply to this context");
  PzPlan pl;
  pz_plan(c, pl);
  const double* H = c.p.hgrid;
  const double c0 = c.p.ggg[0] / (H[0] * H[0]) + c.p.ggg[1] / (H[1] * H[1]) + c.p.ggg[2] / (H[2] * H[2]);
  const double cd[3] = {-0.5 * c.p.ggg[0] / (H[0] * H[0]), -0.5 * c.p.ggg[1] / (H[1] * H[1]),
                        -0.5 * c.p.ggg[2] / (H[2] * H[2])};
  PzArgs a{};
  a.G = G;
  a.P = P;
  a.part = k.part;
  a.sc = k.sc;
  a.nbb = k.nbb;
  a.L = c.p.n1 * (c.cplx ? 2 : 1);
  a.n2 = c.p.n2;
  a.n3 = c.p.n3;
  a.ty = pl.ty;
  a.ytiles = pl.ytiles;
  a.nslot = pl.nslot;
  a.ng = k.ng;
  a.a0 = (float)c0;
  a.a1 = (float)cd[0];
  a.a2 = (float)cd[1];
  a.a3 = (float)cd[2];
  a.b1 = (float)(cd[0] / c0);
  a.b2 = (float)(cd[1] / c0);
  a.b3 = (float)(cd[2] / c0);
  a.first = first;
  a.threads = pl.thr_mom;
  a.status = c.d_status;
  a.polls = c.wait_polls >= 0 ? (uint32_t)c.wait_polls : kWaitPolls;
  RS_CHECK(((uintptr_t)G % 16) == 0 && ((uintptr_t)P % 16) == 0, RSDFT_ERR_ARG, "fused preconditioner: unaligned bands");
  static int nsm = 0;
  if (!nsm) RS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.device));
  const long long items = (long long)k.nbb * pl.ytiles;
  const int grid = (int)std::min<long long>(items, nsm);
  const int ncp = c.cplx ? 2 : 1;
  const int ngr = a.L / 4;
  const int ngs = (ngr == 32 || ngr == 16) ? ngr : 0;
  Blk kz = k;
  kz.nch = pl.ytiles;
  ProfScope ps(c, "pc");
  switch (c.p.mloop) {
    case 1:
      RS_TRY((pz_dispatch<1, true>(c, a, pl.smem_mom, grid, ncp, ngs, pl.thr_mom)));
      k_pcz_sc<1><<<(k.nbb + 127) / 128, 128, 0, c.stream>>>(kz, c0, c.p.dv, first);
      c.launches++;
      RS_TRY((pz_dispatch<1, false>(c, a, pl.smem_upd, grid, ncp, ngs, pl.thr_upd)));
      break;
    case 2:
      RS_TRY((pz_dispatch<2, true>(c, a, pl.smem_mom, grid, ncp, ngs, pl.thr_mom)));
      k_pcz_sc<2><<<(k.nbb + 127) / 128, 128, 0, c.stream>>>(kz, c0, c.p.dv, first);
      c.launches++;
      RS_TRY((pz_dispatch<2, false>(c, a, pl.smem_upd, grid, ncp, ngs, pl.thr_upd)));
      break;
    default:
      RS_TRY((pz_dispatch<3, true>(c, a, pl.smem_mom, grid, ncp, ngs, pl.thr_mom)));
      k_pcz_sc<3><<<(k.nbb + 127) / 128, 128, 0, c.stream>>>(kz, c0, c.p.dv, first);
      c.launches++;
      RS_TRY((pz_dispatch<3, false>(c, a, pl.smem_upd, grid, ncp, ngs, pl.thr_upd)));
      break;
  }
  return check_launch("pc");
}

}  // namespace rsdft
