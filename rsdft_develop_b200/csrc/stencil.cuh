// Pieces shared by the real-build hpsi stencil (hpsi_stream.cu) and its host side (hpsi.cu).
#pragma once
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

// named barrier over the compute threads, OR-reducing a flag
__device__ __forceinline__ bool bar_or(int flag, int nthreads) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, 1, %2, q;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"((uint32_t)flag), "r"((uint32_t)nthreads)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Lane traits of the real stencils: W consecutive x points per thread, held as W/2 pairs.
template <typename T> struct Lanes;
// FP32: 4 x points per thread as two float2 pairs, packed arithmetic
template <> struct Lanes<float> {
  using P2 = float2;
  using U = float4;
  static constexpr int W = 4;
  static constexpr bool packed = true;
  static __device__ __forceinline__ P2 fma(P2 c, P2 a, P2 b) { return __ffma2_rn(c, a, b); }
  static __device__ __forceinline__ P2 add(P2 a, P2 b) { return __fadd2_rn(a, b); }
  static __device__ __forceinline__ P2 mul(P2 a, P2 b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ P2 dup(float c) { return make_float2(c, c); }
  static __device__ __forceinline__ P2 mk(float x, float y) { return make_float2(x, y); }
  static __device__ __forceinline__ P2 pair(const U& u, int j) {
    return j == 0 ? make_float2(u.x, u.y) : make_float2(u.z, u.w);
  }
  static __device__ __forceinline__ U join(const P2 (&p)[2]) { return make_float4(p[0].x, p[0].y, p[1].x, p[1].y); }
  static __device__ __forceinline__ void split(const U& u, float* w) {
    w[0] = u.x;
    w[1] = u.y;
    w[2] = u.z;
    w[3] = u.w;
  }
  static __device__ __forceinline__ float dot4(const float* u, const float* c) {
    const float4 a = *reinterpret_cast<const float4*>(u), b = *reinterpret_cast<const float4*>(c);
    return fmaf(a.x, b.x, fmaf(a.y, b.y, fmaf(a.z, b.z, a.w * b.w)));
  }
};
// FP64: 2 x points per thread as one double2 pair, scalar arithmetic
template <> struct Lanes<double> {
  using P2 = double2;
  using U = double2;
  static constexpr int W = 2;
  static constexpr bool packed = false;
  static __device__ __forceinline__ P2 fma(P2 c, P2 a, P2 b) {
    return make_double2(::fma(c.x, a.x, b.x), ::fma(c.y, a.y, b.y));
  }
  static __device__ __forceinline__ P2 add(P2 a, P2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ P2 mul(P2 a, P2 b) { return make_double2(a.x * b.x, a.y * b.y); }
  static __device__ __forceinline__ P2 dup(double c) { return make_double2(c, c); }
  static __device__ __forceinline__ P2 mk(double x, double y) { return make_double2(x, y); }
  static __device__ __forceinline__ P2 pair(const U& u, int) { return u; }
  static __device__ __forceinline__ U join(const P2 (&p)[1]) { return p[0]; }
  static __device__ __forceinline__ void split(const U& u, double* w) {
    w[0] = u.x;
    w[1] = u.y;
  }
  static __device__ __forceinline__ double dot4(const double* u, const double* c) {
    const double2 a0 = *reinterpret_cast<const double2*>(u), a1 = *reinterpret_cast<const double2*>(u + 2);
    const double2 b0 = *reinterpret_cast<const double2*>(c), b1 = *reinterpret_cast<const double2*>(c + 2);
    return ::fma(a0.x, b0.x, ::fma(a0.y, b0.y, ::fma(a1.x, b1.x, a1.y * b1.y)));
  }
};

template <typename T>
__device__ __forceinline__ typename Lanes<T>::U ldu(const T* p) {
  return *reinterpret_cast<const typename Lanes<T>::U*>(p);
}

template <typename T, int MD>
struct StArgs {
  const T* psi;
  T* out;
  long long ld;
  const T* vloc;
  int n1, n2, n3;
  int tile_y, tz;
  int bx, nact, nthr_c;      // threads along x; active threads; threads per CTA (x32)
  int stage_elems, vl_elems;
  int nst;                   // plane stages in the ring
  T c0;
  T cx[MD], cy[MD], cz[MD];
  const int* rec_rowptr;     // per point: records [rowptr[i], rowptr[i+1])
  const int* rec_pt;         // record -> grid point
  const int* rec_g;          // record -> atom group
  const T* rec_u;            // record -> uV values of the group's projectors [pg]
  int pg;
  const T* coef;             // c_b[g*pg + p], band stride ldc
  int ldc;
  unsigned* status;
  // record ring: each plane's record segment is bulk-copied into shared memory ahead of use
  // (rec_slots == 0: records are read from global memory directly)
  int rec_slots, rec_cap, rec_slot_bytes;
  // persistent CTAs: work items (band, y-tile, z-chunk)
  int ytiles, zch, nb;
};

constexpr int kRecSlotsMax = 3;

// Shared-memory carve of the streaming stencil (host and device agree through smem_layout):
// [S stages: plane rows + V_loc tile][2 nonlocal plane buffers][coefficient row]
// [barriers: S stage, kRecSlotsMax record][kRecSlotsMax record headers][record slots]
struct StLayout {
  size_t nlb, coef, bars, hdr, rec, total;  // byte offsets
};
template <typename T>
__host__ __device__ inline StLayout smem_layout(int S, int stage_elems, int vl_elems, int ldc, int rec_slots,
                                                int rec_slot_bytes) {
  StLayout L;
  L.nlb = sizeof(T) * (size_t)S * (stage_elems + vl_elems);
  L.coef = L.nlb + (ldc > 0 ? sizeof(T) * 2 * (size_t)vl_elems : 0);
  L.bars = L.coef + sizeof(T) * (size_t)((ldc + 15) / 16) * 16;
  L.bars = (L.bars + 15) / 16 * 16;
  L.hdr = L.bars + sizeof(uint64_t) * (size_t)(S + kRecSlotsMax);
  L.hdr = (L.hdr + 15) / 16 * 16;
  L.rec = L.hdr + 16 * (size_t)kRecSlotsMax;
  L.rec = (L.rec + 127) / 128 * 128;
  L.total = L.rec + (size_t)rec_slots * rec_slot_bytes;
  return L;
}

constexpr uint32_t kWaitPolls = 1u << 22;

// persistent streaming stencil (hpsi_stream.cu): autotuned configuration and launch
template <typename T, int MD>
int launch_stencil_stream(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef,
                          const T* vloc_override, double c0_shift);
// warp-specialised streaming stencil + V_loc (hpsi_ws.cu); the nonlocal term is added afterwards
template <typename T, int MD>
int launch_stencil_ws(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* vloc_override,
                      double c0_shift);
// complex-build form (interleaved (re, im) bands, Bloch-phase zcoef taps); nonlocal afterwards
template <typename T, int MD>
int launch_stencil_ws_c(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb);
// largest record segment of one (plane, y-tile) for y-tiles of tile_y rows (cached per tile_y)
int record_segment_max(Ctx& c, int tile_y);

}  // namespace rsdft
