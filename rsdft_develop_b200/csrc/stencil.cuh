// Pieces shared by the real-build hpsi stencil kernels (FP64 and packed-FP32).
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

template <typename T, int MD>
struct StArgs {
  const T* psi;
  T* out;
  long long ld;
  const T* vloc;
  int n1, n2, n3;
  int tile_y, tz;
  int bx, nact, nthr_c;      // threads along x; active compute threads; compute threads (x32)
  int stage_elems, vl_elems, nl_elems;
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
  // record ring: each plane's record segment is bulk-copied into shared memory rec_slots-1
  // planes ahead (rec_slots == 0: records are read from global memory directly)
  int rec_slots, rec_cap, rec_cap_rp, rec_slot_bytes;
};

constexpr int kRecSlotsMax = 3;

// Shared-memory carve of the stencil kernels (host and device agree through smem_layout):
// [S stages: plane rows + V_loc tile][S2 nonlocal plane buffers][coefficient row]
// [barriers: S stage, S2 nl-full, S2 nl-empty, kRecSlotsMax rec-full][kRecSlotsMax headers][record slots]
struct StLayout {
  size_t nlbuf, coef, bars, hdr, rec, total;  // byte offsets
};
template <typename T>
__host__ __device__ inline StLayout smem_layout(int S, int S2, int stage_elems, int vl_elems, int nl_elems, int ldc,
                                                int rec_slots, int rec_slot_bytes) {
  StLayout L;
  L.nlbuf = sizeof(T) * (size_t)S * (stage_elems + vl_elems);
  L.coef = L.nlbuf + sizeof(T) * (size_t)S2 * nl_elems;
  L.bars = L.coef + sizeof(T) * (size_t)((ldc + 15) / 16) * 16;
  L.bars = (L.bars + 15) / 16 * 16;
  L.hdr = L.bars + sizeof(uint64_t) * (size_t)(S + 2 * S2 + kRecSlotsMax);
  L.hdr = (L.hdr + 15) / 16 * 16;
  L.rec = L.hdr + 16 * (size_t)kRecSlotsMax;
  L.rec = (L.rec + 127) / 128 * 128;
  L.total = L.rec + (size_t)rec_slots * rec_slot_bytes;
  return L;
}

constexpr uint32_t kWaitPolls = 1u << 22;
constexpr int kNLW = 2;  // nonlocal warps per CTA
constexpr int kRB = 8;   // records in flight per nonlocal thread


// Nonlocal warps (kNLW of them, threads nthr_c .. nthr_c + 32 kNLW - 1): for each plane of
// the CTA's z-range, the projector scatter  nl(r) = sum_a sum_p uV_a,p(r) c_b[a,p]  at every
// point r of the tile, written into the plane buffer of an S2-deep ring (handed over through
// nlfull/nlempty).  The records are kept per point (CSR: rec_rowptr over grid points, then
// atom rec_g and uV values rec_u per record), so each nonlocal thread sums the records of its
// own points -- every buffer entry is written once, no atomics, no clearing.  A plane's row
// pointers and records are two contiguous segments; with a record ring the first nonlocal
// thread bulk-copies both rec_slots-1 planes ahead (ranges rounded out to 4 entries for the
// 16-byte copy rule; the tables carry padding for that).  Without a ring, or for a segment
// larger than a slot, the records are read from global memory.
template <typename T, int MD>
__device__ __forceinline__ T nl_point(const StArgs<T, MD>& a, const T* coef_s, const int* g, const T* u, int r0,
                                      int r1) {
  T v = T(0);
  for (int r = r0; r < r1; ++r) {
    const T* cg = coef_s + g[r] * a.pg;
    const T* uu = u + (size_t)r * a.pg;
    for (int q = 0; q < a.pg; ++q) v += uu[q] * cg[q];
  }
  return v;
}

template <typename T, int MD, int S2>
__device__ __forceinline__ void nl_warps(const StArgs<T, MD>& a, T* nlbuf, const T* coef_s, uint64_t* nlfull,
                                         uint64_t* nlempty, uint64_t* recfull, int4* rechdr, unsigned char* recbuf,
                                         int tid, int nthr_c, int z0, int zend, int y0, int ty_valid) {
  const int n1 = a.n1, n2 = a.n2;
  const int lt = tid - nthr_c;  // 0 .. 32*kNLW-1
  const int npl = zend - z0;
  const int npts = ty_valid * n1;
  const int RS = a.rec_slots;
  const int cap = a.rec_cap;      // records per slot
  const int capr = a.rec_cap_rp;  // row-pointer entries per slot
  int issued = 0;                 // planes whose copies the producer (lt == 0) has issued
  // slot: [row pointers: capr ints][atoms: cap ints][uV: cap * pg T]
  // header: {direct, row-pointer offset, record base (first staged record), -}
  auto rec_issue = [&](int pi) {
    const int slot = pi % RS;
    const int base = ((z0 + pi) * n2 + y0) * n1;
    const int rs = __ldg(a.rec_rowptr + base), re = __ldg(a.rec_rowptr + base + npts);
    const int a0 = rs & ~3, a1 = (re + 3) & ~3, n = a1 - a0;
    const int b0 = base & ~3, b1 = (base + npts + 1 + 3) & ~3, nr = b1 - b0;
    int4 h;
    uint32_t bytes = 0;
    if (n <= cap && nr <= capr) {
      h = make_int4(0, base - b0, a0, 0);
      bytes = (uint32_t)nr * 4u + (uint32_t)n * (4u + (uint32_t)(a.pg * sizeof(T)));
    } else {
      h = make_int4(1, 0, 0, 0);
    }
    rechdr[slot] = h;
    mbar_arrive_expect_tx(&recfull[slot], bytes);
    if (bytes) {
      unsigned char* sb = recbuf + (size_t)slot * a.rec_slot_bytes;
      bulk_g2s(sb, a.rec_rowptr + b0, (uint32_t)nr * 4u, &recfull[slot]);
      bulk_g2s(sb + (size_t)capr * 4, a.rec_g + a0, (uint32_t)n * 4u, &recfull[slot]);
      bulk_g2s(sb + (size_t)(capr + cap) * 4, a.rec_u + (size_t)a0 * a.pg, (uint32_t)((size_t)n * a.pg * sizeof(T)),
               &recfull[slot]);
    }
  };
  auto give_up = [&](int from) {
    atomicOr(a.status, DEV_WAIT_TIMEOUT);
    if (lt == 0)
      for (int q = from; q < issued; ++q) mbar_wait_bounded(&recfull[q % RS], (uint32_t)((q / RS) & 1), kWaitPolls);
  };
  if (RS > 0 && lt == 0)
    for (; issued < RS - 1 && issued < npl; ++issued) rec_issue(issued);
  for (int pi = 0; pi < npl; ++pi) {
    const int slot = pi % S2;
    if (pi >= S2) {
      const bool ok = mbar_wait_bounded(&nlempty[slot], (uint32_t)(((pi / S2) - 1) & 1), kWaitPolls);
      if (!ok) {
        give_up(pi);
        return;
      }
    }
    T* nl = nlbuf + (size_t)slot * a.nl_elems;
    const int base = ((z0 + pi) * n2 + y0) * n1;
    bool direct = true;
    if (RS > 0) {
      // all nonlocal threads are past plane pi-1, whose record slot the producer refills
      asm volatile("bar.sync 2, %0;" ::"r"(32 * kNLW) : "memory");
      if (lt == 0 && issued < npl) {
        fence_proxy_async_smem();
        rec_issue(issued);
        ++issued;
      }
      const int rslot = pi % RS;
      if (!mbar_wait_bounded(&recfull[rslot], (uint32_t)((pi / RS) & 1), kWaitPolls)) {
        give_up(pi);
        return;
      }
      const int4 h = rechdr[rslot];
      if (h.x == 0) {
        direct = false;
        const unsigned char* sb = recbuf + (size_t)rslot * a.rec_slot_bytes;
        const int* srp = reinterpret_cast<const int*>(sb) + h.y;
        const int* sg = reinterpret_cast<const int*>(sb + (size_t)capr * 4);
        const T* su = reinterpret_cast<const T*>(sb + (size_t)(capr + cap) * 4);
        for (int e = lt; e < npts; e += 32 * kNLW) nl[e] = nl_point(a, coef_s, sg, su, srp[e] - h.z, srp[e + 1] - h.z);
      }
    }
    if (direct) {
      for (int e = lt; e < npts; e += 32 * kNLW)
        nl[e] = nl_point(a, coef_s, a.rec_g, a.rec_u, __ldg(a.rec_rowptr + base + e), __ldg(a.rec_rowptr + base + e + 1));
    }
    __syncwarp();
    if ((lt & 31) == 0) mbar_arrive(&nlfull[slot]);
  }
}

// packed-FP32 kernel (hpsi_f32.cu): its largest block at its register count, and its launch
template <int MD, int S, int S2>
int stencil_f32_block_limit(int* max_threads);
template <int MD, int S, int S2>
int launch_stencil_f32(const StArgs<float, MD>& a, dim3 grid, dim3 block, size_t smem, cudaStream_t st);

}  // namespace rsdft
