// Many-band hpsi stencil for the real8 (Gamma) build: H psi = T psi + V_loc psi + V_NL psi.
//
// Reference semantics (restated, not translated):
//   kinetic + V_loc  src/kinetic/d_kinetic_sol_module.f90:244-292 (Md=6 star stencil,
//                    (coef_lap0 + V_loc) on the centre, periodic halo src/bc/bcset_3_module.f90)
//   nonlocal         src/ps_nloc_mr_module.f90:1159-1258 (scatter psi(JJP) += uVk * sum Dij uVunk);
//                    the coefficient rows c_b = D (dV uV^T psi_b) come from the gather kernel.
//
// Design (B200): persistent CTAs walk work items (band, y-tile, z-chunk); a work item is an
// N1 x TY column of one band streamed along z.
//  * Thread 0 bulk-copies (TMA engine, cp.async.bulk + mbarrier) each xy-plane of the column
//    with an Md-deep periodic y halo and its V_loc tile into an S-deep ring, and each plane's
//    nonlocal records (grid point, atom, uV per record) into an RS-deep ring, a few planes
//    ahead and across work-item boundaries.
//  * Every thread owns W consecutive x points (one 16-byte shared-memory load) on R rows: x taps
//    wrap inside the staged full row, y taps read neighbouring staged rows, z taps are pushed
//    into 2*Md+1 rotating register accumulators (each plane is read once from HBM).  FP32 runs
//    on float2 pairs with sm_100's packed FMA/ADD/MUL; FP64 on scalars with the same pairing.
//  * Nonlocal term (the fused form; by default hpsi adds it with a scatter kernel after this
//    kernel instead): one step ahead, all threads of the CTA share out the next plane's staged
//    records evenly, each adding uV . c_b[atom] into that plane's buffer with a shared-memory
//    atomic; on the next step each thread takes its own points' sums with one vector load per
//    row and clears them (two buffers by plane parity; the per-step barrier orders both).
//  * R (rows per thread: register blocking against occupancy) is picked per shape by timing
//    both variants on the first call (autotuning).
// Thread 0 issues the plane stages and thread 32 the record segments.  All waits are bounded;
// a timeout sets the device status word (RSDFT_ERR_TIMEOUT) and every CTA drains its own
// copies in flight before it exits.
#include "stencil.cuh"

namespace rsdft {

namespace {

// z push for rotation slot S: acc[S] += t, acc[S -+ m] += cz_m v, then emit slot S - Md
template <typename T, int MD, int R, int S>
__device__ __forceinline__ void zpush(typename Lanes<T>::P2 (&acc)[2 * MD + 1][R][Lanes<T>::W / 2],
                                      const typename Lanes<T>::P2 (&v)[R][Lanes<T>::W / 2],
                                      const typename Lanes<T>::P2 (&t)[R][Lanes<T>::W / 2], const T (&cz)[MD],
                                      bool fin, T* orow, int n1, const bool (&rowok)[R]) {
  using L = Lanes<T>;
  constexpr int P = L::W / 2;
  constexpr int NQ = 2 * MD + 1;
  if constexpr (S < NQ) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) acc[S][r][j] = L::add(acc[S][r][j], t[r][j]);
#pragma unroll
    for (int m = 1; m <= MD; ++m) {
      const auto c = L::dup(cz[m - 1]);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) {
          acc[(S - m + NQ) % NQ][r][j] = L::fma(c, v[r][j], acc[(S - m + NQ) % NQ][r][j]);
          acc[(S + m) % NQ][r][j] = L::fma(c, v[r][j], acc[(S + m) % NQ][r][j]);
        }
    }
    constexpr int FS = (S + NQ - MD) % NQ;
    if (fin) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (rowok[r]) *reinterpret_cast<typename L::U*>(orow + (size_t)r * n1) = L::join(acc[FS][r]);
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) acc[FS][r][j] = L::dup(T(0));
  }
}

#define RS_ZP_CASE(S_)                                          \
  case S_:                                                      \
    zpush<T, MD, R, S_>(acc, v, t, a.cz, fin, orow, n1, rowok); \
    break;

// Work item w: band w / (ytiles * zch), then y-tile and z-chunk.
struct Item {
  int band, y0, z0, zend, ty_valid, nplanes;
};
template <typename T, int MD>
__device__ __forceinline__ Item item_of(const StArgs<T, MD>& a, int w) {
  Item it;
  const int per_band = a.ytiles * a.zch;
  it.band = w / per_band;
  const int r = w - it.band * per_band;
  const int yt = r % a.ytiles, zc = r / a.ytiles;
  it.y0 = yt * a.tile_y;
  it.z0 = zc * a.tz;
  it.zend = min(it.z0 + a.tz, a.n3);
  it.ty_valid = min(a.tile_y, a.n2 - it.y0);
  it.nplanes = (it.zend - it.z0) + 2 * MD;
  return it;
}

}  // namespace

// R rows per thread: R = 2 keeps 2W points per thread (1 CTA of 8 warps per SM, up to 255
// registers); R = 1 keeps W (2 CTAs per SM at <= 128 registers).
template <typename T, int MD, int R>
__global__ void __launch_bounds__(256, 3 - R) k_stencil_stream(const StArgs<T, MD> a) {
  using L = Lanes<T>;
  using P2 = typename L::P2;
  constexpr int W = L::W;
  constexpr int P = W / 2;
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + W - 1) / W;  // W-wide chunks of x halo per side
  extern __shared__ __align__(128) unsigned char smem[];
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const int S = a.nst;  // plane stages in the ring
  const StLayout Ly = smem_layout<T>(S, a.stage_elems, a.vl_elems, a.ldc, a.rec_slots, a.rec_slot_bytes);
  T* stages = reinterpret_cast<T*>(smem);
  const int sstride = a.stage_elems + a.vl_elems;
  T* nlb = reinterpret_cast<T*>(smem + Ly.nlb);  // [2][vl_elems] nonlocal sums of a plane, by parity
  T* coef_s = reinterpret_cast<T*>(smem + Ly.coef);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + Ly.bars);
  uint64_t* recfull = bar + S;
  int4* rechdr = reinterpret_cast<int4*>(smem + Ly.hdr);
  unsigned char* recbuf = smem + Ly.rec;

  const int tid = threadIdx.x;
  const int nthr = a.nthr_c;
  const bool active = tid < a.nact;
  const int tx = tid % a.bx, ty = tid / a.bx;
  const int x0 = tx * W;
  const int yl = ty * R;
  const int yrow = active ? yl : 0;
  const int rows = a.tile_y + 2 * MD;
  const bool nl_on = a.rec_rowptr != nullptr;
  const int RS = a.rec_slots;
  const int cap = a.rec_cap;
  const int nwork = a.ytiles * a.zch * a.nb;

  if (tid == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
    for (int s = 0; s < RS; ++s) mbar_init(&recfull[s], 1);
    fence_mbar_init();
  }
  if (nl_on)  // the plane buffers start at zero; every reader clears what it has read
    for (int i = tid; i < 2 * a.vl_elems; i += blockDim.x) nlb[i] = T(0);
  __syncthreads();

  // ---- producer state (thread 0): plane stages and record segments, issued ahead ----
  long long gis = 0;            // plane stages issued
  int pw = blockIdx.x, pq = 0;  // stage cursor: work item, plane within it
  Item pit;
  if (pw < nwork) pit = item_of<T, MD>(a, pw);
  long long gri = 0;             // record segments issued
  int rw = blockIdx.x, rpi = 0;  // record cursor: work item, interior plane
  Item rit;
  if (rw < nwork) rit = item_of<T, MD>(a, rw);
  int pf_rs = 0, pf_re = 0;  // row pointers of the record cursor's plane (loaded a step ahead)
  auto rec_base = [&]() { return ((rit.z0 + rpi) * n2 + rit.y0) * n1; };
  // thread 0 issues the plane stages, thread kRecTid (another warp) the record segments, so
  // that neither warp carries both producers' work into the per-step barrier
  const int rec_tid = blockDim.x > 32 ? 32 : 0;
  if (tid == rec_tid && nl_on && RS > 0 && rw < nwork) {
    pf_rs = __ldg(a.rec_rowptr + rec_base());
    pf_re = __ldg(a.rec_rowptr + rec_base() + rit.ty_valid * n1);
  }
  auto issue_stage = [&]() {
    const int q = pq;
    const T* src = a.psi + (long long)pit.band * a.ld;
    const int zg = pmod(pit.z0 - MD + q, n3);
    const int slot = (int)(gis % S);
    T* st = stages + (size_t)slot * sstride;
    uint64_t* br = &bar[slot];
    const int p = pit.z0 - MD + q;
    const bool inch = p >= pit.z0 && p < pit.zend;
    const uint32_t bytes = (uint32_t)((size_t)rows * n1 * sizeof(T)) +
                           (inch ? (uint32_t)((size_t)pit.ty_valid * n1 * sizeof(T)) : 0u);
    mbar_arrive_expect_tx(br, bytes);
    int r = 0;
    while (r < rows) {
      const int gy = pmod(pit.y0 - MD + r, n2);
      const int len = min(rows - r, n2 - gy);
      bulk_g2s(st + (size_t)r * n1, src + ((size_t)zg * n2 + gy) * n1, (uint32_t)((size_t)len * n1 * sizeof(T)),
               br);
      r += len;
    }
    if (inch)
      bulk_g2s(st + a.stage_elems, a.vloc + ((size_t)p * n2 + pit.y0) * n1,
               (uint32_t)((size_t)pit.ty_valid * n1 * sizeof(T)), br);
    ++gis;
    if (++pq == pit.nplanes) {
      pq = 0;
      pw += gridDim.x;
      if (pw < nwork) pit = item_of<T, MD>(a, pw);
    }
  };
  // slot: [points: cap ints][atoms: cap ints][uV: cap * pg values]
  // header: {direct, first record of the segment within the slot, records, -}
  auto issue_rec = [&]() {
    const int slot = (int)(gri % RS);
    const int rs = pf_rs, re = pf_re;
    const int a0 = rs & ~3, a1 = (re + 3) & ~3, n = a1 - a0;
    int4 h;
    uint32_t bytes = 0;
    if (n <= cap) {
      h = make_int4(0, rs - a0, re - rs, 0);
      bytes = (uint32_t)n * (8u + (uint32_t)(a.pg * sizeof(T)));
    } else {
      h = make_int4(1, 0, 0, 0);
    }
    rechdr[slot] = h;
    mbar_arrive_expect_tx(&recfull[slot], bytes);
    if (bytes) {
      unsigned char* sb = recbuf + (size_t)slot * a.rec_slot_bytes;
      bulk_g2s(sb, a.rec_pt + a0, (uint32_t)n * 4u, &recfull[slot]);
      bulk_g2s(sb + (size_t)cap * 4, a.rec_g + a0, (uint32_t)n * 4u, &recfull[slot]);
      bulk_g2s(sb + (size_t)cap * 8, a.rec_u + (size_t)a0 * a.pg, (uint32_t)((size_t)n * a.pg * sizeof(T)),
               &recfull[slot]);
    }
    ++gri;
    if (++rpi == rit.zend - rit.z0) {
      rpi = 0;
      rw += gridDim.x;
      if (rw < nwork) rit = item_of<T, MD>(a, rw);
    }
    if (rw < nwork) {  // prefetch the next segment's row pointers; used at the next issue
      pf_rs = __ldg(a.rec_rowptr + rec_base());
      pf_re = __ldg(a.rec_rowptr + rec_base() + rit.ty_valid * n1);
    }
  };

  // x-window chunk offsets (wrapped once per thread)
  int xl[NCH], xr[NCH];
#pragma unroll
  for (int ch = 1; ch <= NCH; ++ch) {
    xl[ch - 1] = pmod(x0 - W * ch, n1);
    xr[ch - 1] = pmod(x0 + W * ch, n1);
  }

  long long gq = 0;   // plane stages consumed
  long long grc = 0;  // record segments consumed
  bool aborted = false;
  bool cur_direct = true, next_direct = true;  // nonlocal sums of the current / next plane from global memory
  typename L::U zero_u;  // a zero vector of W values
  {
    P2 zp[P];
#pragma unroll
    for (int j = 0; j < P; ++j) zp[j] = L::dup(T(0));
    zero_u = L::join(zp);
  }
  P2 acc[NQ][R][P];
  for (int w = blockIdx.x; w < nwork && !aborted; w += gridDim.x) {
    const Item it = item_of<T, MD>(a, w);
    const T* coef_g = a.coef + (long long)it.band * a.ldc;
    T* dst = a.out + (long long)it.band * a.ld;
    // the previous item ended with a barrier over all threads: the coefficient row is free,
    // and its first use comes Md steps (and barriers) later
    if (nl_on)
      for (int i = tid; i < a.ldc; i += blockDim.x) coef_s[i] = coef_g[i];
    bool rowok[R];
#pragma unroll
    for (int r = 0; r < R; ++r) rowok[r] = active && (yl + r) < it.ty_valid;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) acc[q][r][j] = L::dup(T(0));

    for (int q = 0; q < it.nplanes; ++q) {
      if (tid == 0) {
        fence_proxy_async_smem();  // slots refilled below were read through the generic proxy
        while (gis < gq + S && pw < nwork) issue_stage();
      }
      if (tid == rec_tid && nl_on && RS > 0) {
        fence_proxy_async_smem();
        while (gri < grc + RS && rw < nwork) issue_rec();
      }
      const int slot = (int)(gq % S);
      bool ok = mbar_wait_bounded(&bar[slot], (uint32_t)((gq / S) & 1), kWaitPolls);
      const T* pl = stages + (size_t)slot * sstride;
      const T* prow = pl + (size_t)(yrow + MD) * n1;  // own first row
      const int p = it.z0 - MD + q;
      const bool inch = p >= it.z0 && p < it.zend;
      P2 v[R][P], t[R][P];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const auto c = ldu(prow + (size_t)r * n1 + x0);
#pragma unroll
        for (int j = 0; j < P; ++j) {
          v[r][j] = L::pair(c, j);
          t[r][j] = L::dup(T(0));
        }
      }
      if (inch) {
        // centre: (c0 + V_loc) psi
        const P2 c0 = L::dup(a.c0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const auto vl = ldu(pl + a.stage_elems + (size_t)(yrow + r) * n1 + x0);
#pragma unroll
          for (int j = 0; j < P; ++j) t[r][j] = L::mul(L::add(c0, L::pair(vl, j)), v[r][j]);
        }
        // x taps: window w[-W NCH .. W NCH + W - 1] of the staged (periodic) row
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const T* row = prow + (size_t)r * n1;
          T wv[(2 * NCH + 1) * W];
#pragma unroll
          for (int j = 0; j < P; ++j) {
            wv[W * NCH + 2 * j] = v[r][j].x;
            wv[W * NCH + 2 * j + 1] = v[r][j].y;
          }
#pragma unroll
          for (int ch = 1; ch <= NCH; ++ch) {
            L::split(ldu(row + xl[ch - 1]), wv + W * (NCH - ch));
            L::split(ldu(row + xr[ch - 1]), wv + W * (NCH + ch));
          }
          constexpr int C = W * NCH;  // index of x0 in wv
#pragma unroll
          for (int m = 1; m <= MD; ++m) {
            const T cm = a.cx[m - 1];
            if (!L::packed || (m & 1) == 0) {
#pragma unroll
              for (int j = 0; j < P; ++j) {
                const P2 lp = L::mk(wv[C + 2 * j - m], wv[C + 2 * j + 1 - m]);
                const P2 rp = L::mk(wv[C + 2 * j + m], wv[C + 2 * j + 1 + m]);
                t[r][j] = L::fma(L::dup(cm), L::add(lp, rp), t[r][j]);
              }
            } else {
#pragma unroll
              for (int j = 0; j < P; ++j) {
                t[r][j].x = ::fma(cm, wv[C + 2 * j - m] + wv[C + 2 * j + m], t[r][j].x);
                t[r][j].y = ::fma(cm, wv[C + 2 * j + 1 - m] + wv[C + 2 * j + 1 + m], t[r][j].y);
              }
            }
          }
        }
        // y taps: rows yl-MD .. yl+R-1+MD of the stage; the own rows come from v
#pragma unroll
        for (int dy = -MD; dy < R + MD; ++dy) {
          P2 rv[P];
          if (dy >= 0 && dy < R) {
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = v[(dy >= 0 && dy < R) ? dy : 0][j];
          } else {
            const auto c = ldu(prow + (ptrdiff_t)dy * n1 + x0);
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = L::pair(c, j);
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int m = dy > r ? dy - r : r - dy;
            if (m >= 1 && m <= MD) {
              const P2 cm = L::dup(a.cy[(m >= 1 && m <= MD ? m : 1) - 1]);
#pragma unroll
              for (int j = 0; j < P; ++j) t[r][j] = L::fma(cm, rv[j], t[r][j]);
            }
          }
        }
        // nonlocal term of the own points: sums prepared one step earlier (or from global
        // memory when that plane's records did not fit a slot)
        if (nl_on) {
          const int base = (p * n2 + it.y0) * n1;
          T* nlp = nlb + (size_t)(p & 1) * a.vl_elems;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            if (!rowok[r]) continue;
            const int e0 = (yl + r) * n1 + x0;
            T nv[W];
            if (!cur_direct) {
              L::split(ldu(nlp + e0), nv);
              *reinterpret_cast<typename L::U*>(nlp + e0) = zero_u;  // cleared for plane p + 2
            } else {
              int rp[W + 1];
#pragma unroll
              for (int i = 0; i <= W; ++i) rp[i] = __ldg(a.rec_rowptr + base + e0 + i);
#pragma unroll
              for (int i = 0; i < W; ++i) {
                T acc_nl = T(0);
                for (int k = rp[i]; k < rp[i + 1]; ++k) {
                  const int g = __ldg(a.rec_g + k);
                  for (int qq = 0; qq < a.pg; ++qq)
                    acc_nl = ::fma(__ldg(a.rec_u + (size_t)k * a.pg + qq), coef_s[g * a.pg + qq], acc_nl);
                }
                nv[i] = acc_nl;
              }
            }
#pragma unroll
            for (int j = 0; j < P; ++j) t[r][j] = L::add(t[r][j], L::mk(nv[2 * j], nv[2 * j + 1]));
          }
        }
      }
      // the next plane's nonlocal sums, record by record over all threads, into its buffer
      bool consumed = false;
      if (nl_on && p + 1 >= it.z0 && p + 1 < it.zend) {
        bool nd = true;
        if (RS > 0) {
          const int rslot = (int)(grc % RS);
          ok = mbar_wait_bounded(&recfull[rslot], (uint32_t)((grc / RS) & 1), kWaitPolls) && ok;
          consumed = true;
          const int4 h = rechdr[rslot];
          if (h.x == 0) {
            nd = false;
            const unsigned char* sb = recbuf + (size_t)rslot * a.rec_slot_bytes;
            const int* spt = reinterpret_cast<const int*>(sb) + h.y;
            const int* sg = reinterpret_cast<const int*>(sb + (size_t)cap * 4) + h.y;
            const T* su = reinterpret_cast<const T*>(sb + (size_t)cap * 8) + (size_t)h.y * a.pg;
            T* nln = nlb + (size_t)((p + 1) & 1) * a.vl_elems;
            const int nbase = ((p + 1) * n2 + it.y0) * n1;
            for (int e = tid; e < h.z; e += blockDim.x) {
              const int g = sg[e];
              T v;
              if (a.pg == 4) {
                v = L::dot4(su + (size_t)e * 4, coef_s + g * 4);
              } else {
                v = T(0);
                for (int qq = 0; qq < a.pg; ++qq) v = ::fma(su[(size_t)e * a.pg + qq], coef_s[g * a.pg + qq], v);
              }
              atomicAdd(nln + (spt[e] - nbase), v);
            }
          }
        }
        next_direct = nd;
      }
      const int zo = p - MD;
      const bool fin = zo >= it.z0 && zo < it.zend;
      T* orow = dst + ((size_t)(fin ? zo : 0) * n2 + (it.y0 + yl)) * n1 + x0;
      switch (q % NQ) {
        RS_ZP_CASE(0) RS_ZP_CASE(1) RS_ZP_CASE(2) RS_ZP_CASE(3) RS_ZP_CASE(4) RS_ZP_CASE(5)
        RS_ZP_CASE(6) RS_ZP_CASE(7) RS_ZP_CASE(8) RS_ZP_CASE(9) RS_ZP_CASE(10) RS_ZP_CASE(11)
        RS_ZP_CASE(12)
        default: break;
      }
      ++gq;
      if (consumed) ++grc;
      cur_direct = next_direct;
      if (bar_or(!ok, nthr)) {
        aborted = true;
        break;
      }
    }
  }
  // drain copies still in flight before the CTA's shared memory is released (each producer its
  // own ring, only the phases not consumed: a slot's barrier has moved on past earlier ones)
  if (aborted && tid == 0) {
    atomicOr(a.status, DEV_WAIT_TIMEOUT);
    for (long long q = gq; q < gis; ++q) mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
  }
  if (aborted && tid == rec_tid)
    for (long long q = grc; q < gri; ++q) mbar_wait_bounded(&recfull[q % RS], (uint32_t)((q / RS) & 1), kWaitPolls);
  if (aborted) __syncthreads();
}

// One variant (rows per thread R) configured for this grid and launched on the library stream.
template <typename T, int MD, int R>
static int launch_variant(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef,
                          const T* vloc_override, double c0_shift) {
  constexpr bool F32 = std::is_same<T, float>::value;
  constexpr int W = Lanes<T>::W;
  // stages: 1 CTA per SM (R = 2) or 2 (R = 1); fewer when the record ring needs the room
  constexpr int SMAX = R == 2 ? (F32 ? 6 : 5) : (F32 ? 4 : 3);
  constexpr int CTAS = 3 - R;  // CTAs per SM
  const size_t budget = CTAS == 1 ? 225 * 1024 : 112 * 1024;
  auto kern = k_stencil_stream<T, MD, R>;
  static int max_block = 0, nsm = 0;  // one per template instantiation
  if (!max_block) {
    cudaFuncAttributes fa{};
    RS_CUDA(cudaFuncGetAttributes(&fa, kern));
    max_block = fa.maxThreadsPerBlock;
    int dev = 0;
    RS_CUDA(cudaGetDevice(&dev));
    RS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)budget));
  }
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  RS_CHECK(n1 % W == 0 && ld % W == 0, RSDFT_ERR_UNSUPPORTED, "hpsi needs N1 and ld multiples of %d", W);
  const int bx = n1 / W;
  const int max_c = std::min(256, (max_block / 32) * 32);
  RS_CHECK(bx <= max_c, RSDFT_ERR_UNSUPPORTED, "N1=%d needs %d threads per row; this build allows %d", n1, bx, max_c);
  int by = std::max(1, max_c / bx);
  by = std::min(by, (n2 + R - 1) / R);
  const int nthr = ((bx * by + 31) / 32) * 32;
  const int tile_y = by * R;
  const int rows = tile_y + 2 * MD;
  constexpr int AL = 128 / (int)sizeof(T);  // 128-byte aligned stage sections
  auto rnd = [&](int e) { return ((e + AL - 1) / AL) * AL; };
  const int stage_elems = rnd(rows * n1), vl_elems = rnd(tile_y * n1);
  const bool nl_on = c.nl.nproj > 0 && coef != nullptr;
  const int ldc = nl_on ? c.nl.ngroups * c.nl.pg : 0;
  int S = SMAX;
  int rec_slots = 0, rec_cap = 0, rec_slot_bytes = 0;
  if (nl_on) {
    rec_cap = ((record_segment_max(c, tile_y) + 6) + 3) / 4 * 4;
    rec_slot_bytes = (int)(((size_t)rec_cap * (8 + c.nl.pg * sizeof(T)) + 127) / 128 * 128);
    for (int st = SMAX; st >= 3 && rec_slots == 0; --st)
      for (int rs = kRecSlotsMax; rs >= 2; --rs)
        if (smem_layout<T>(st, stage_elems, vl_elems, ldc, rs, rec_slot_bytes).total <= budget) {
          rec_slots = rs;
          S = st;
          break;
        }
  }
  const size_t smem = smem_layout<T>(S, stage_elems, vl_elems, ldc, rec_slots, rec_slot_bytes).total;
  {  // configuration of this variant, readable through rsdft_gpu_profile_get
    const std::string pre = std::string(F32 ? "stencil" : "stencil64") + (R == 1 ? "_r1" : "_r2");
    c.tune_ms[pre + "_stages"] = S;
    c.tune_ms[pre + "_rec_slots"] = rec_slots;
    c.tune_ms[pre + "_smem_kb"] = smem / 1024.0;
  }
  RS_CHECK(smem <= budget, RSDFT_ERR_UNSUPPORTED, "stencil stages (%zu B) exceed shared memory", smem);
  const int ytiles = (n2 + tile_y - 1) / tile_y;
  int zch = 1;
  while ((long long)ytiles * zch * nb < (long long)nsm * CTAS && n3 / (zch * 2) >= 16) zch *= 2;
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;

  StArgs<T, MD> a{};
  a.psi = psi;
  a.out = out;
  a.ld = (long long)ld;
  a.vloc = vloc_override
               ? vloc_override
               : (F32 ? (const T*)c.vloc32.as<float>() : (const T*)c.vloc64.as<double>()) + (size_t)s * c.ng;
  a.n1 = n1;
  a.n2 = n2;
  a.n3 = n3;
  a.tile_y = tile_y;
  a.tz = tz;
  a.bx = bx;
  a.nact = bx * by;
  a.nthr_c = nthr;
  a.stage_elems = stage_elems;
  a.vl_elems = vl_elems;
  a.nst = S;
  a.c0 = (T)(c.p.coef_lap0 + c.kp[k].const_k2 + c0_shift);
  for (int m = 0; m < MD; ++m) {
    a.cx[m] = (T)c.p.coef_lap[0][m];
    a.cy[m] = (T)c.p.coef_lap[1][m];
    a.cz[m] = (T)c.p.coef_lap[2][m];
  }
  a.rec_rowptr = nl_on ? c.nl.rec_rowptr.as<int>() : nullptr;
  a.rec_pt = nl_on ? c.nl.rec_pt.as<int>() : nullptr;
  a.rec_g = nl_on ? c.nl.rec_g.as<int>() : nullptr;
  a.rec_u = nl_on ? (F32 ? (const T*)c.nl.perk[k].ru32.as<float>() : (const T*)c.nl.perk[k].ru64.as<double>())
                  : nullptr;
  a.pg = c.nl.pg;
  a.coef = coef;
  a.ldc = ldc;
  a.status = c.d_status;
  a.rec_slots = rec_slots;
  a.rec_cap = rec_cap;
  a.rec_slot_bytes = rec_slot_bytes;
  a.ytiles = ytiles;
  a.zch = zch;
  a.nb = nb;
  const int nwork = ytiles * zch * nb;
  const int grid = std::min(nwork, nsm * CTAS);
  kern<<<grid, nthr, smem, c.stream>>>(a);
  c.launches++;
  return check_launch("hpsi_stencil");
}

// Autotuned launch: the first call for a (grid, band count, projector, precision) shape times
// each variant (rows per thread 1 or 2: occupancy against per-thread register blocking) with
// CUDA events on the library stream and keeps the faster; every timed run computes the full
// result, so the output of the call is complete either way.
template <typename T, int MD>
int launch_stencil_stream(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef,
                          const T* vloc_override, double c0_shift) {
  const bool nl_on = c.nl.nproj > 0 && coef != nullptr;
  const double e = (double)sizeof(T);
  // algorithmic bytes: read psi + write H psi per band; V_loc, the record tables once
  const double alg_bytes = e * (2.0 * (double)c.ng * nb + (double)c.ng) +
                           (nl_on ? 4.0 * (double)(c.ng + 1) + (4.0 + e * c.nl.pg) * c.nl.ftotal : 0.0);
  const int nbc = nb >= 64 ? 64 : (nb >= 8 ? 8 : 1);  // band-count class
  const long long key =
      ((((long long)c.p.n1 * 1024 + c.p.n2) * 1024 + c.p.n3) * 256 + nbc * 2 + (nl_on ? 1 : 0)) * 2 +
      (sizeof(T) == 8 ? 1 : 0);
  auto it = c.stencil_tune.find(key);
  if (it == c.stencil_tune.end()) {
    float best = 1e30f;
    int pick = 2;
    cudaEvent_t e0, e1;
    RS_CUDA(cudaEventCreate(&e0));
    RS_CUDA(cudaEventCreate(&e1));
    for (int r = 1; r <= 2; ++r) {
      for (int rep = 0; rep < 2; ++rep) {
        RS_CUDA(cudaEventRecord(e0, c.stream));
        const int st = r == 1 ? launch_variant<T, MD, 1>(c, k, s, psi, out, ld, nb, coef, vloc_override, c0_shift)
                              : launch_variant<T, MD, 2>(c, k, s, psi, out, ld, nb, coef, vloc_override, c0_shift);
        if (st != 0) break;
        RS_CUDA(cudaEventRecord(e1, c.stream));
        RS_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        RS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep == 1) {
          c.tune_ms[std::string(sizeof(T) == 8 ? "stencil64" : "stencil") + (r == 1 ? "_tune_r1" : "_tune_r2")] = ms;
          if (ms < best) {
            best = ms;
            pick = r;
          }
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    it = c.stencil_tune.emplace(key, pick).first;
  }
  ProfScope ps(c, "hpsi_stencil", alg_bytes);
  if (it->second == 1) return launch_variant<T, MD, 1>(c, k, s, psi, out, ld, nb, coef, vloc_override, c0_shift);
  return launch_variant<T, MD, 2>(c, k, s, psi, out, ld, nb, coef, vloc_override, c0_shift);
}

template int launch_stencil_stream<float, 6>(Ctx&, int, int, const float*, float*, size_t, int, const float*,
                                            const float*, double);
template int launch_stencil_stream<float, 4>(Ctx&, int, int, const float*, float*, size_t, int, const float*,
                                            const float*, double);
template int launch_stencil_stream<double, 6>(Ctx&, int, int, const double*, double*, size_t, int, const double*,
                                             const double*, double);
template int launch_stencil_stream<double, 4>(Ctx&, int, int, const double*, double*, size_t, int, const double*,
                                             const double*, double);

}  // namespace rsdft
