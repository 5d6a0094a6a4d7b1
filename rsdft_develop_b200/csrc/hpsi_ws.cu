// Many-band hpsi stencil for the real8 (Gamma) build, warp-specialised form:
//   H psi = (coef_lap0 + const_k2 + V_loc) psi + sum_d sum_m coef_lap(d, m) (psi[i - m e_d] + psi[i + m e_d])
//
// Reference semantics (restated, not translated): src/kinetic/d_kinetic_sol_module.f90:244-292
// (Md-deep star stencil, (coef_lap0 + V_loc) on the centre) with the periodic halo of
// src/bc/bcset_3_module.f90:15-151.  The nonlocal term is added after this kernel by the scatter
// in hpsi.cu (src/ps_nloc_mr_module.f90:1159-1258).
//
// Design (B200, sm_100a):
//  * Persistent CTAs, one per SM, walk work items (band, y-tile, z-chunk).  An item is an
//    N1 x TY column of one band streamed along z; a plane stage holds the TY + 2 Md rows of the
//    column (periodic y halo) and the item's V_loc rows.
//  * One producer warp (lane 0) fills an S-deep ring of plane stages with bulk copies (TMA
//    engine, cp.async.bulk completing on a per-slot "full" mbarrier) and refills a slot once
//    every consumer warp has released it on the slot's "empty" mbarrier.  There is no CTA-wide
//    barrier per plane: consumer warps drift up to S planes apart.
//  * Consumer threads own W consecutive x points (one 16-byte shared-memory load: 4 FP32 or
//    2 FP64) on R rows: x taps come from a window of 16-byte loads of the staged (periodic) row,
//    y taps from the neighbouring staged rows, z taps are pushed into 2 Md + 1 rotating register
//    accumulators, so each plane is read from HBM once.  FP32 arithmetic runs on float2 pairs
//    with sm_100's packed FFMA2/FADD2/FMUL2 wherever the pair is register-aligned (y, z, centre
//    and even-m x taps).
//  * Ring bookkeeping uses 32-bit slot/round counters (no division in the plane loop).
//  * All waits are bounded.  A thread whose wait gives up sets the device status word
//    (RSDFT_ERR_TIMEOUT) and a shared abort flag; every waiter polls the flag and leaves, and
//    the producer waits for each slot's last bulk copy before its CTA exits.
#include "stencil.cuh"

namespace rsdft {

namespace {

template <typename T, int MD>
struct WsArgs {
  const T* psi;
  T* out;
  long long ld;
  const T* vloc;
  int n1, n2, n3;
  int tile_y, tz, ytiles, zch, nb;
  int bx, by, ncw;      // threads per row, row groups per tile, consumer warps
  int stage_elems;      // (tile_y + 2 MD) rows of n1, rounded to 128 bytes
  int vl_elems;         // tile_y rows of n1, rounded to 128 bytes
  int nst;              // stages in the ring
  int bar_off;          // byte offset of the barriers
  int vlg;              // real build: 1 = V_loc rows read from global memory (L2), not staged
  T c0;
  T cx[MD], cy[MD], cz[MD];
  T cs[3][MD];          // complex build: coef_nabk(d, m); zcoef_kin(d, +m) = c_d(m) - i cs[d][m]
  unsigned* status;
  uint32_t polls;       // polls of a bounded wait before it gives up
};

struct WsItem {
  int band, y0, z0, zend, ty_valid, nplanes;
};

template <typename T, int MD>
__device__ __forceinline__ WsItem ws_item(const WsArgs<T, MD>& a, int w) {
  WsItem it;
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

// Bounded wait that also leaves when another thread of the CTA has given up.
__device__ __forceinline__ bool ws_wait(uint64_t* bar, uint32_t parity, const volatile int* abort_flag,
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


// Compile-time loop: f(std::integral_constant<int, I>) for I in [B, E).
template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>());
    sfor<B + 1, E>(f);
  }
}

// 16-byte shared-memory loads at a 32-bit shared address, with a compile-time byte offset
// (an immediate of the load) or a run-time address.
template <typename T> struct Sld;
template <> struct Sld<float> {
  template <int OFF>
  static __device__ __forceinline__ float4 at(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a), "n"(OFF));
    return v;
  }
  static __device__ __forceinline__ float4 rt(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
  }
};
template <> struct Sld<double> {
  template <int OFF>
  static __device__ __forceinline__ double2 at(uint32_t a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2+%3];" : "=d"(v.x), "=d"(v.y) : "r"(a), "n"(OFF));
    return v;
  }
  static __device__ __forceinline__ double2 rt(uint32_t a) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(a));
    return v;
  }
};

// z push for rotation slot S: acc[S] += t (own x/y/centre terms, interior planes only),
// acc[S -+ m] += cz_m v; acc[S + MD] was emitted at the previous step, so its first term is a
// product, not a sum.  Then acc[S - MD] holds a finished output plane.
template <typename T, int MD, int R, int S>
__device__ __forceinline__ void ws_zpush(typename Lanes<T>::P2 (&acc)[2 * MD + 1][R][Lanes<T>::W / 2],
                                         const typename Lanes<T>::P2 (&v)[R][Lanes<T>::W / 2],
                                         const typename Lanes<T>::P2 (&t)[R][Lanes<T>::W / 2],
                                         const typename Lanes<T>::P2 (&czp)[MD], bool inch, bool fin, T* orow, int n1,
                                         const bool (&rowok)[R]) {
  using L = Lanes<T>;
  constexpr int P = L::W / 2;
  constexpr int NQ = 2 * MD + 1;
  if constexpr (S < NQ) {
    if (inch) {
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) acc[S][r][j] = L::add(acc[S][r][j], t[r][j]);
    }
#pragma unroll
    for (int m = 1; m <= MD; ++m) {
      const auto c = czp[m - 1];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) {
          acc[(S - m + NQ) % NQ][r][j] = L::fma(c, v[r][j], acc[(S - m + NQ) % NQ][r][j]);
          if (m == MD)
            acc[(S + m) % NQ][r][j] = L::mul(c, v[r][j]);
          else
            acc[(S + m) % NQ][r][j] = L::fma(c, v[r][j], acc[(S + m) % NQ][r][j]);
        }
    }
    constexpr int FS = (S + NQ - MD) % NQ;
    if (fin) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (rowok[r]) *reinterpret_cast<typename L::U*>(orow + (size_t)r * n1) = L::join(acc[FS][r]);
    }
  }
}

#define RS_WS_CASE(S_)                                                    \
  case S_:                                                                \
    ws_zpush<T, MD, R, S_>(acc, v, t, czp, inch, fin, orow, n1, rowok); \
    break;

}  // namespace

// R rows per thread.  R = 2: 8 points per FP32 thread, 26 rotating float2 accumulators per
// row pair; one CTA of up to 12 warps per SM.
// N1C > 0 fixes the row length at compile time, so every shared-memory offset of the plane
// step is an immediate; N1C = 0 reads it from the arguments.
template <typename T, int MD, int R, int N1C>
__global__ void __launch_bounds__(384, 1) k_stencil_ws(const WsArgs<T, MD> a) {
  using L = Lanes<T>;
  using P2 = typename L::P2;
  constexpr int W = L::W;
  constexpr int P = W / 2;
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + W - 1) / W;  // W-wide chunks of x halo per side
  extern __shared__ __align__(128) unsigned char smem[];
  T* stages = reinterpret_cast<T*>(smem);
  const int sstride = a.stage_elems + a.vl_elems;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + a.bar_off);
  uint64_t* empty = full + a.nst;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + a.nst);
  const int S = a.nst;
  const int n1 = N1C > 0 ? N1C : a.n1;
  const int n2 = a.n2, n3 = a.n3;
  const int nwork = a.ytiles * a.zch * a.nb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rows = a.tile_y + 2 * MD;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (uint32_t)a.ncw);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == a.ncw) {
    // ---------------- producer ----------------
    if (lane != 0) return;
    int slot = 0, round = 0;
    int issued = 0;
    bool ab = false;
    for (int w = blockIdx.x; w < nwork && !ab; w += gridDim.x) {
      const WsItem it = ws_item(a, w);
      const T* src = a.psi + (long long)it.band * a.ld;
      for (int q = 0; q < it.nplanes; ++q) {
        if (round > 0 && !ws_wait(&empty[slot], (uint32_t)((round - 1) & 1), abort_flag, a.polls)) {
          ab = true;
          break;
        }
        fence_proxy_async_smem();  // the slot was last read through the generic proxy
        const int p = it.z0 - MD + q;
        const int zg = pmod(p, n3);
        const bool inch = q >= MD && p < it.zend;
        T* st = stages + (size_t)slot * sstride;
        const uint32_t bytes = (uint32_t)((size_t)rows * n1 * sizeof(T)) +
                               (inch && !a.vlg ? (uint32_t)((size_t)it.ty_valid * n1 * sizeof(T)) : 0u);
        mbar_arrive_expect_tx(&full[slot], bytes);
        int r = 0;
        while (r < rows) {
          const int gy = pmod(it.y0 - MD + r, n2);
          const int len = min(rows - r, n2 - gy);
          bulk_g2s(st + (size_t)r * n1, src + ((size_t)zg * n2 + gy) * n1, (uint32_t)((size_t)len * n1 * sizeof(T)),
                   &full[slot]);
          r += len;
        }
        if (inch && !a.vlg)
          bulk_g2s(st + a.stage_elems, a.vloc + ((size_t)p * n2 + it.y0) * n1,
                   (uint32_t)((size_t)it.ty_valid * n1 * sizeof(T)), &full[slot]);
        ++issued;
        if (++slot == S) {
          slot = 0;
          ++round;
        }
      }
    }
    if (ab) {
      *abort_flag = 1;
      atomicOr(a.status, DEV_WAIT_TIMEOUT);
    }
    // Before this thread exits, wait (with the full limit, whatever a.polls says) for the last
    // copy issued into every slot: if consumers gave up, copies may still be in flight, and the
    // CTA's shared memory must outlive them.  On the normal path they have all landed already.
    for (int s = 0; s < S && s < issued; ++s) {
      const int last = ((issued - 1 - s) / S) * S + s;
      for (uint32_t it = 0; it < kWaitPolls; ++it)
        if (mbar_try_wait(&full[s], (uint32_t)((last / S) & 1))) break;
    }
    return;
  }

  // ---------------- consumers ----------------
  const int ct = threadIdx.x;
  const int bx = N1C > 0 ? N1C / W : a.bx;
  const int tx = ct % bx, ty = ct / bx;
  const bool active = ty < a.by;
  const int x0 = tx * W;
  const int yl = (active ? ty : 0) * R;
  // per-thread byte offsets inside a stage: own column (first staged row of the thread's
  // window, yl), x-window chunks (wrapped periodically), V_loc tile
  constexpr uint32_t E = sizeof(T);
  const uint32_t yoff = (uint32_t)yl * (uint32_t)n1 * E;
  const uint32_t off0 = yoff + (uint32_t)x0 * E;
  uint32_t offl[NCH], offr[NCH];
#pragma unroll
  for (int ch = 1; ch <= NCH; ++ch) {
    offl[ch - 1] = yoff + (uint32_t)pmod(x0 - W * ch, n1) * E;
    offr[ch - 1] = yoff + (uint32_t)pmod(x0 + W * ch, n1) * E;
  }
  const uint32_t offv = (uint32_t)a.stage_elems * E + off0;
  const uint32_t sbase0 = smem_u32(stages);
  const uint32_t sstride_b = (uint32_t)sstride * E;
  // row k of the thread's window (k = 0 is staged row yl, its own rows are k = MD .. MD + R - 1)
  auto ldrow = [&](uint32_t base, auto kc) -> typename L::U {
    constexpr int kk = decltype(kc)::value;
    if constexpr (N1C > 0)
      return Sld<T>::template at<kk * N1C * (int)sizeof(T)>(base);
    else
      return Sld<T>::rt(base + (uint32_t)kk * (uint32_t)n1 * E);
  };
  const P2 c0 = L::dup(a.c0);
  P2 cyp[MD], czp[MD];
#pragma unroll
  for (int m = 0; m < MD; ++m) {
    cyp[m] = L::dup(a.cy[m]);
    czp[m] = L::dup(a.cz[m]);
  }
  int slot = 0, round = 0;
  P2 acc[NQ][R][P];
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const WsItem it = ws_item(a, w);
    T* dst = a.out + (long long)it.band * a.ld;
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
      const int p = it.z0 - MD + q;
      const bool inch = q >= MD && p < it.zend;
      // V_loc rows from global memory (L2-resident), issued before the wait so that their
      // latency overlaps it; rows past the tile are not read
      typename L::U vlr[R];
      if (a.vlg && inch) {
        const T* vrow = a.vloc + ((size_t)p * n2 + it.y0 + yl) * n1 + x0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (rowok[r]) vlr[r] = __ldg(reinterpret_cast<const typename L::U*>(vrow + (size_t)r * n1));
          else vlr[r] = typename L::U{};
        }
      }
      if (!ws_wait(&full[slot], (uint32_t)(round & 1), abort_flag, a.polls)) {
        if (!*abort_flag) {
          *abort_flag = 1;
          atomicOr(a.status, DEV_WAIT_TIMEOUT);
        }
        return;
      }
      const uint32_t sb = sbase0 + (uint32_t)slot * sstride_b;
      const uint32_t a0 = sb + off0;
      P2 v[R][P], t[R][P];
      sfor<0, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        const auto u = ldrow(a0, std::integral_constant<int, MD + r>());
#pragma unroll
        for (int j = 0; j < P; ++j) v[r][j] = L::pair(u, j);
      });
      if (inch) {
        // centre: (c0 + V_loc) psi
        const uint32_t av = sb + offv;
        sfor<0, R>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          const auto vl = a.vlg ? vlr[r] : ldrow(av, rc);
#pragma unroll
          for (int j = 0; j < P; ++j) t[r][j] = L::mul(L::add(c0, L::pair(vl, j)), v[r][j]);
        });
        // x taps from the window w[C - W NCH .. C + W NCH + W - 1] of the staged periodic row
        uint32_t al[NCH], ar[NCH];
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
          al[ch] = sb + offl[ch];
          ar[ch] = sb + offr[ch];
        }
        sfor<0, R>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          constexpr std::integral_constant<int, MD + r> kc{};
          T wv[(2 * NCH + 1) * W];
#pragma unroll
          for (int j = 0; j < P; ++j) {
            wv[W * NCH + 2 * j] = v[r][j].x;
            wv[W * NCH + 2 * j + 1] = v[r][j].y;
          }
#pragma unroll
          for (int ch = 1; ch <= NCH; ++ch) {
            L::split(ldrow(al[ch - 1], kc), wv + W * (NCH - ch));
            L::split(ldrow(ar[ch - 1], kc), wv + W * (NCH + ch));
          }
          constexpr int C = W * NCH;
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
        });
        // y taps: window rows k = 0 .. R + 2 MD - 1 (dy = k - MD); the own rows come from v
        sfor<0, R + 2 * MD>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          constexpr int dy = k - MD;
          P2 rv[P];
          if constexpr (dy >= 0 && dy < R) {
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = v[dy][j];
          } else {
            const auto u = ldrow(a0, kc);
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = L::pair(u, j);
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int m = dy > r ? dy - r : r - dy;
            if (m >= 1 && m <= MD) {
              const P2 cm = cyp[(m >= 1 && m <= MD ? m : 1) - 1];
#pragma unroll
              for (int j = 0; j < P; ++j) t[r][j] = L::fma(cm, rv[j], t[r][j]);
            }
          }
        });
      }
      // every shared-memory read of this stage is done: release the slot to the producer
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      if (++slot == S) {
        slot = 0;
        ++round;
      }
      const int zo = p - MD;
      const bool fin = q >= 2 * MD;
      T* orow = dst + ((size_t)(fin ? zo : 0) * n2 + (it.y0 + yl)) * n1 + x0;
      switch (q % NQ) {
        RS_WS_CASE(0) RS_WS_CASE(1) RS_WS_CASE(2) RS_WS_CASE(3) RS_WS_CASE(4) RS_WS_CASE(5)
        RS_WS_CASE(6) RS_WS_CASE(7) RS_WS_CASE(8) RS_WS_CASE(9) RS_WS_CASE(10) RS_WS_CASE(11)
        RS_WS_CASE(12)
        default: break;
      }
    }
  }
}

// Launch configuration: the tile height maximises rows per CTA within the consumer-thread
// limit and splits N2 into equal tiles; z-chunks are added when they balance the persistent
// CTAs' work better than they cost in halo planes.
template <typename T, int MD>
int launch_stencil_ws(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* vloc_override,
                      double c0_shift) {
  constexpr int R = 2;
  constexpr int W = Lanes<T>::W;
  constexpr int MAXW = 12;  // warps per CTA (__launch_bounds__)
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  auto kern = n1 == 64 ? k_stencil_ws<T, MD, R, 64>
              : n1 == 96 ? k_stencil_ws<T, MD, R, 96>
              : n1 == 128 ? k_stencil_ws<T, MD, R, 128> : k_stencil_ws<T, MD, R, 0>;
  static int nsm = 0;  // one per template instantiation of the launcher
  if (!nsm) {
    int dev = 0;
    RS_CUDA(cudaGetDevice(&dev));
    RS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (auto kf : {k_stencil_ws<T, MD, R, 64>, k_stencil_ws<T, MD, R, 96>, k_stencil_ws<T, MD, R, 128>,
                    k_stencil_ws<T, MD, R, 0>})
      RS_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  }
  RS_CHECK(n1 % W == 0 && ld % W == 0, RSDFT_ERR_UNSUPPORTED, "hpsi needs N1 and ld multiples of %d", W);
  RS_CHECK(((uintptr_t)psi % 16) == 0 && ((uintptr_t)out % 16) == 0, RSDFT_ERR_ARG,
           "hpsi needs 16-byte aligned wavefunction blocks");
  const int bx = n1 / W;
  const int maxc = (MAXW - 1) * 32;
  RS_CHECK(bx <= maxc, RSDFT_ERR_UNSUPPORTED, "N1=%d needs %d threads per row; this build allows %d", n1, bx, maxc);
  int by_max = std::max(1, std::min(maxc / bx, (n2 + R - 1) / R));
  const int ytiles = (n2 + by_max * R - 1) / (by_max * R);
  const int by = (n2 + ytiles * R - 1) / (ytiles * R);
  const int tile_y = by * R;
  const int ncw = (bx * by + 31) / 32;
  const int rows = tile_y + 2 * MD;
  constexpr int AL = 128 / (int)sizeof(T);
  auto rnd = [&](int e) { return ((e + AL - 1) / AL) * AL; };
  // V_loc rows staged with the plane, or (vlg) read by the consumers from L2, which leaves the
  // shared memory to more psi planes in flight
  const int vlg = c.stencil_vloc_global && !vloc_override ? 1 : 0;
  const int stage_elems = rnd(rows * n1), vl_elems = vlg ? 0 : rnd(tile_y * n1);
  const size_t stage_bytes = sizeof(T) * (size_t)(stage_elems + vl_elems);
  const size_t budget = 227 * 1024 - 256;
  int S = (int)std::min<size_t>(vlg ? 12 : 8, budget / stage_bytes);
  RS_CHECK(S >= 2, RSDFT_ERR_UNSUPPORTED, "stencil stage (%zu B) does not fit shared memory twice", stage_bytes);
  const int bar_off = (int)(stage_bytes * S);
  const size_t smem = (size_t)bar_off + 16 * (size_t)S + 16;
  // z-chunks: balance of items over the CTAs against the extra halo planes a chunk costs
  // (a halo plane costs about a quarter of an interior plane: the z push only)
  int zch = 1;
  double best = -1.0;
  for (int zc = 1; zc <= 8; zc *= 2) {
    const int tz = (n3 + zc - 1) / zc;
    if (zc > 1 && tz < 2 * MD) break;
    const long long items = (long long)ytiles * ((n3 + tz - 1) / tz) * nb;
    const long long grid = std::min<long long>(items, nsm);
    const double bal = (double)items / (double)(grid * ((items + grid - 1) / grid));
    const double score = bal * (double)tz / (tz + 0.25 * 2 * MD);
    if (score > best + 1e-3) {
      best = score;
      zch = zc;
    }
  }
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;

  WsArgs<T, MD> a{};
  a.psi = psi;
  a.out = out;
  a.ld = (long long)ld;
  const bool f32 = std::is_same<T, float>::value;
  a.vloc = vloc_override ? vloc_override
                         : (f32 ? (const T*)c.vloc32.as<float>() : (const T*)c.vloc64.as<double>()) + (size_t)s * c.ng;
  a.n1 = n1;
  a.n2 = n2;
  a.n3 = n3;
  a.tile_y = tile_y;
  a.tz = tz;
  a.ytiles = ytiles;
  a.zch = zch;
  a.nb = nb;
  a.bx = bx;
  a.by = by;
  a.ncw = ncw;
  a.stage_elems = stage_elems;
  a.vl_elems = vl_elems;
  a.nst = S;
  a.bar_off = bar_off;
  a.vlg = vlg;
  a.c0 = (T)(c.p.coef_lap0 + c.kp[k].const_k2 + c0_shift);
  for (int m = 0; m < MD; ++m) {
    a.cx[m] = (T)c.p.coef_lap[0][m];
    a.cy[m] = (T)c.p.coef_lap[1][m];
    a.cz[m] = (T)c.p.coef_lap[2][m];
  }
  a.status = c.d_status;
  a.polls = c.wait_polls >= 0 ? (uint32_t)c.wait_polls : kWaitPolls;
  {  // configuration, readable through rsdft_gpu_profile_get
    const std::string pre = f32 ? "stencil" : "stencil64";
    c.tune_ms[pre + "_stages"] = S;
    c.tune_ms[pre + "_tile_y"] = tile_y;
    c.tune_ms[pre + "_warps"] = ncw + 1;
    c.tune_ms[pre + "_zchunks"] = zch;
    c.tune_ms[pre + "_smem_kb"] = smem / 1024.0;
  }
  const long long nwork = (long long)ytiles * zch * nb;
  const int grid = (int)std::min<long long>(nwork, nsm);
  const double e = (double)sizeof(T);
  ProfScope ps(c, "hpsi_stencil", e * (2.0 * (double)c.ng * nb + (double)c.ng));
  kern<<<grid, (ncw + 1) * 32, smem, c.stream>>>(a);
  c.launches++;
  return check_launch("hpsi_stencil");
}

template int launch_stencil_ws<float, 6>(Ctx&, int, int, const float*, float*, size_t, int, const float*, double);
template int launch_stencil_ws<float, 4>(Ctx&, int, int, const float*, float*, size_t, int, const float*, double);
template int launch_stencil_ws<double, 6>(Ctx&, int, int, const double*, double*, size_t, int, const double*, double);
template int launch_stencil_ws<double, 4>(Ctx&, int, int, const double*, double*, size_t, int, const double*, double);

// ---------------------------------------------------------------------------------------------
// complex16 (Bloch k-point) form.  H u(i) = (coef_lap0 + const_k2 + V_loc) u(i)
//   + sum_d sum_m [ zcoef(d, m) u(i + m e_d) + conj(zcoef(d, m)) u(i - m e_d) ],
//   zcoef(d, m) = coef_lap(d, m) - i coef_nabk(d, m)
// (src/kinetic/d_kinetic_sol_module.f90:144-200, the z_ module on complex arrays;
// src/kinetic/kinetic_module.f90:155-159), periodic wrap of u.  Same producer / ring / z-push
// design as the real kernel; a grid point is an interleaved (re, im) pair held as one register
// pair, so z u = (c, c) u + (s, -s) swap(u) and conj(z) u = (c, c) u + (-s, s) swap(u) are two
// packed FMAs (FP32) per update; x taps use the pair sums c (u+ + u-) and -i s (u+ - u-).
// The nonlocal term is added by the complex scatter kernel afterwards.
// ---------------------------------------------------------------------------------------------
namespace {

template <typename T, int MD, int R, int S>
__device__ __forceinline__ void ws_zpush_c(typename Lanes<T>::P2 (&acc)[2 * MD + 1][R][Lanes<T>::W / 2],
                                           const typename Lanes<T>::P2 (&v)[R][Lanes<T>::W / 2],
                                           const typename Lanes<T>::P2 (&t)[R][Lanes<T>::W / 2],
                                           const WsArgs<T, MD>& a, bool inch, bool fin, T* orow, int rowlen,
                                           const bool (&rowok)[R]) {
  using L = Lanes<T>;
  using P2 = typename L::P2;
  constexpr int P = L::W / 2;
  constexpr int NQ = 2 * MD + 1;
  if constexpr (S < NQ) {
    if (inch) {
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) acc[S][r][j] = L::add(acc[S][r][j], t[r][j]);
    }
    P2 sw[R][P];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int j = 0; j < P; ++j) sw[r][j] = L::mk(v[r][j].y, v[r][j].x);
#pragma unroll
    for (int m = 1; m <= MD; ++m) {
      const P2 cc = L::dup(a.cz[m - 1]);
      const T sn = a.cs[2][m - 1];
      const P2 sp = L::mk(sn, -sn), sm = L::mk(-sn, sn);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int j = 0; j < P; ++j) {
          // plane p is the +m neighbour of output p - m (zcoef) and the -m neighbour of p + m
          P2& lo = acc[(S - m + NQ) % NQ][r][j];
          lo = L::fma(sp, sw[r][j], L::fma(cc, v[r][j], lo));
          P2& hi = acc[(S + m) % NQ][r][j];
          if (m == MD)
            hi = L::fma(sm, sw[r][j], L::mul(cc, v[r][j]));
          else
            hi = L::fma(sm, sw[r][j], L::fma(cc, v[r][j], hi));
        }
    }
    constexpr int FS = (S + NQ - MD) % NQ;
    if (fin) {
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (rowok[r]) *reinterpret_cast<typename L::U*>(orow + (size_t)r * rowlen) = L::join(acc[FS][r]);
    }
  }
}

#define RS_WSC_CASE(S_)                                                        \
  case S_:                                                                     \
    ws_zpush_c<T, MD, R, S_>(acc, v, t, a, inch, fin, orow, rowlen, rowok);    \
    break;

}  // namespace

// N1C: complex points per row fixed at compile time (0: run time).  Rows of a stage hold 2 n1
// reals; each consumer thread owns W reals (W / 2 complex points) on R rows.
template <typename T, int MD, int R, int N1C>
__global__ void __launch_bounds__(384, 1) k_stencil_ws_c(const WsArgs<T, MD> a) {
  using L = Lanes<T>;
  using P2 = typename L::P2;
  constexpr int W = L::W;
  constexpr int P = W / 2;                       // complex points per thread and row
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (2 * MD + W - 1) / W;      // W-real chunks of x halo per side
  extern __shared__ __align__(128) unsigned char smem[];
  T* stages = reinterpret_cast<T*>(smem);
  const int sstride = a.stage_elems + a.vl_elems;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + a.bar_off);
  uint64_t* empty = full + a.nst;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + a.nst);
  const int S = a.nst;
  const int n1 = N1C > 0 ? N1C : a.n1;
  const int rowlen = 2 * n1;                     // reals per row
  const int n2 = a.n2, n3 = a.n3;
  const int nwork = a.ytiles * a.zch * a.nb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rows = a.tile_y + 2 * MD;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], (uint32_t)a.ncw);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == a.ncw) {
    // ---------------- producer ----------------
    if (lane != 0) return;
    int slot = 0, round = 0;
    int issued = 0;
    bool ab = false;
    for (int w = blockIdx.x; w < nwork && !ab; w += gridDim.x) {
      const WsItem it = ws_item(a, w);
      const T* src = a.psi + (long long)it.band * a.ld;
      for (int q = 0; q < it.nplanes; ++q) {
        if (round > 0 && !ws_wait(&empty[slot], (uint32_t)((round - 1) & 1), abort_flag, a.polls)) {
          ab = true;
          break;
        }
        fence_proxy_async_smem();
        const int p = it.z0 - MD + q;
        const int zg = pmod(p, n3);
        const bool inch = q >= MD && p < it.zend;
        T* st = stages + (size_t)slot * sstride;
        const uint32_t bytes = (uint32_t)((size_t)rows * rowlen * sizeof(T)) +
                               (inch ? (uint32_t)((size_t)it.ty_valid * n1 * sizeof(T)) : 0u);
        mbar_arrive_expect_tx(&full[slot], bytes);
        int r = 0;
        while (r < rows) {
          const int gy = pmod(it.y0 - MD + r, n2);
          const int len = min(rows - r, n2 - gy);
          bulk_g2s(st + (size_t)r * rowlen, src + ((size_t)zg * n2 + gy) * rowlen,
                   (uint32_t)((size_t)len * rowlen * sizeof(T)), &full[slot]);
          r += len;
        }
        if (inch)
          bulk_g2s(st + a.stage_elems, a.vloc + ((size_t)p * n2 + it.y0) * n1,
                   (uint32_t)((size_t)it.ty_valid * n1 * sizeof(T)), &full[slot]);
        ++issued;
        if (++slot == S) {
          slot = 0;
          ++round;
        }
      }
    }
    if (ab) {
      *abort_flag = 1;
      atomicOr(a.status, DEV_WAIT_TIMEOUT);
    }
    for (int s = 0; s < S && s < issued; ++s) {
      const int last = ((issued - 1 - s) / S) * S + s;
      for (uint32_t it = 0; it < kWaitPolls; ++it)
        if (mbar_try_wait(&full[s], (uint32_t)((last / S) & 1))) break;
    }
    return;
  }

  // ---------------- consumers ----------------
  const int ct = threadIdx.x;
  const int bx = N1C > 0 ? 2 * N1C / W : a.bx;
  const int tx = ct % bx, ty = ct / bx;
  const bool active = ty < a.by;
  const int x0 = tx * W;      // first real of the thread in the row
  const int xc = x0 / 2;      // its first complex point
  const int yl = (active ? ty : 0) * R;
  constexpr uint32_t E = sizeof(T);
  const uint32_t yoff = (uint32_t)yl * (uint32_t)rowlen * E;
  const uint32_t off0 = yoff + (uint32_t)x0 * E;
  uint32_t offl[NCH], offr[NCH];
#pragma unroll
  for (int ch = 1; ch <= NCH; ++ch) {
    offl[ch - 1] = yoff + (uint32_t)pmod(x0 - W * ch, rowlen) * E;
    offr[ch - 1] = yoff + (uint32_t)pmod(x0 + W * ch, rowlen) * E;
  }
  const uint32_t offv = (uint32_t)a.stage_elems * E + (uint32_t)yl * (uint32_t)n1 * E + (uint32_t)xc * E;
  const uint32_t sbase0 = smem_u32(stages);
  const uint32_t sstride_b = (uint32_t)sstride * E;
  auto ldrow = [&](uint32_t base, auto kc) -> typename L::U {
    constexpr int kk = decltype(kc)::value;
    if constexpr (N1C > 0)
      return Sld<T>::template at<kk * 2 * N1C * (int)sizeof(T)>(base);
    else
      return Sld<T>::rt(base + (uint32_t)kk * (uint32_t)rowlen * E);
  };
  int slot = 0, round = 0;
  P2 acc[NQ][R][P];
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const WsItem it = ws_item(a, w);
    T* dst = a.out + (long long)it.band * a.ld;
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
      if (!ws_wait(&full[slot], (uint32_t)(round & 1), abort_flag, a.polls)) {
        if (!*abort_flag) {
          *abort_flag = 1;
          atomicOr(a.status, DEV_WAIT_TIMEOUT);
        }
        return;
      }
      const uint32_t sb = sbase0 + (uint32_t)slot * sstride_b;
      const uint32_t a0 = sb + off0;
      const int p = it.z0 - MD + q;
      const bool inch = q >= MD && p < it.zend;
      P2 v[R][P], t[R][P];
      sfor<0, R>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        const auto u = ldrow(a0, std::integral_constant<int, MD + r>());
#pragma unroll
        for (int j = 0; j < P; ++j) v[r][j] = L::pair(u, j);
      });
      if (inch) {
        // centre: (c0 + V_loc) u, V_loc real (one value per complex point)
        const T* vl = reinterpret_cast<const T*>(smem + (sb - sbase0) + offv);
#pragma unroll
        for (int r = 0; r < R; ++r)
#pragma unroll
          for (int j = 0; j < P; ++j) t[r][j] = L::mul(L::dup(a.c0 + vl[(size_t)r * n1 + j]), v[r][j]);
        // x taps: complex neighbours at +-m are reals +-2m away in the staged periodic row
        uint32_t al[NCH], ar[NCH];
#pragma unroll
        for (int ch = 0; ch < NCH; ++ch) {
          al[ch] = sb + offl[ch];
          ar[ch] = sb + offr[ch];
        }
        sfor<0, R>([&](auto rc) {
          constexpr int r = decltype(rc)::value;
          constexpr std::integral_constant<int, MD + r> kc{};
          T wv[(2 * NCH + 1) * W];
#pragma unroll
          for (int j = 0; j < P; ++j) {
            wv[W * NCH + 2 * j] = v[r][j].x;
            wv[W * NCH + 2 * j + 1] = v[r][j].y;
          }
#pragma unroll
          for (int ch = 1; ch <= NCH; ++ch) {
            L::split(ldrow(al[ch - 1], kc), wv + W * (NCH - ch));
            L::split(ldrow(ar[ch - 1], kc), wv + W * (NCH + ch));
          }
          constexpr int C = W * NCH;
#pragma unroll
          for (int m = 1; m <= MD; ++m) {
            const P2 cc = L::dup(a.cx[m - 1]);
            const T sn = a.cs[0][m - 1];
#pragma unroll
            for (int j = 0; j < P; ++j) {
              const P2 up = L::mk(wv[C + 2 * j + 2 * m], wv[C + 2 * j + 2 * m + 1]);
              const P2 um = L::mk(wv[C + 2 * j - 2 * m], wv[C + 2 * j - 2 * m + 1]);
              const P2 sp = L::add(up, um);
              const P2 dp = L::fma(L::dup(T(-1)), um, up);
              t[r][j] = L::fma(cc, sp, t[r][j]);
              t[r][j].x = ::fma(sn, dp.y, t[r][j].x);
              t[r][j].y = ::fma(-sn, dp.x, t[r][j].y);
            }
          }
        });
        // y taps: row dy is the +m neighbour (zcoef) of own row r when dy > r, the -m one
        // (conj(zcoef)) when dy < r
        sfor<0, R + 2 * MD>([&](auto kc) {
          constexpr int k = decltype(kc)::value;
          constexpr int dy = k - MD;
          P2 rv[P];
          if constexpr (dy >= 0 && dy < R) {
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = v[dy][j];
          } else {
            const auto u = ldrow(a0, kc);
#pragma unroll
            for (int j = 0; j < P; ++j) rv[j] = L::pair(u, j);
          }
          P2 sw[P];
#pragma unroll
          for (int j = 0; j < P; ++j) sw[j] = L::mk(rv[j].y, rv[j].x);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int m = dy - r;
            const int am = m > 0 ? m : -m;
            if (am >= 1 && am <= MD) {
              const P2 cc = L::dup(a.cy[(am >= 1 && am <= MD ? am : 1) - 1]);
              const T sn = a.cs[1][(am >= 1 && am <= MD ? am : 1) - 1];
              const P2 sq = m > 0 ? L::mk(sn, -sn) : L::mk(-sn, sn);
#pragma unroll
              for (int j = 0; j < P; ++j) t[r][j] = L::fma(sq, sw[j], L::fma(cc, rv[j], t[r][j]));
            }
          }
        });
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[slot]);
      if (++slot == S) {
        slot = 0;
        ++round;
      }
      const int zo = p - MD;
      const bool fin = q >= 2 * MD;
      T* orow = dst + ((size_t)(fin ? zo : 0) * n2 + (it.y0 + yl)) * rowlen + x0;
      switch (q % NQ) {
        RS_WSC_CASE(0) RS_WSC_CASE(1) RS_WSC_CASE(2) RS_WSC_CASE(3) RS_WSC_CASE(4) RS_WSC_CASE(5)
        RS_WSC_CASE(6) RS_WSC_CASE(7) RS_WSC_CASE(8) RS_WSC_CASE(9) RS_WSC_CASE(10) RS_WSC_CASE(11)
        RS_WSC_CASE(12)
        default: break;
      }
    }
  }
}

// Complex-build launch: the same tiling rule as the real kernel on rows of 2 n1 reals.
template <typename T, int MD>
int launch_stencil_ws_c(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb) {
  constexpr int R = 2;
  constexpr int W = Lanes<T>::W;
  constexpr int MAXW = 12;
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  auto kern = n1 == 64 ? k_stencil_ws_c<T, MD, R, 64> : k_stencil_ws_c<T, MD, R, 0>;
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    RS_CUDA(cudaGetDevice(&dev));
    RS_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (auto kf : {k_stencil_ws_c<T, MD, R, 64>, k_stencil_ws_c<T, MD, R, 0>})
      RS_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  }
  const int rowlen = 2 * n1;
  RS_CHECK(rowlen % W == 0 && ld % W == 0 && n1 % W == 0, RSDFT_ERR_UNSUPPORTED,
           "complex hpsi needs N1 a multiple of %d and ld a multiple of %d reals", W, W);
  RS_CHECK(((uintptr_t)psi % 16) == 0 && ((uintptr_t)out % 16) == 0, RSDFT_ERR_ARG,
           "hpsi needs 16-byte aligned wavefunction blocks");
  const int bx = rowlen / W;
  const int maxc = (MAXW - 1) * 32;
  RS_CHECK(bx <= maxc, RSDFT_ERR_UNSUPPORTED, "N1=%d needs %d threads per row; this build allows %d", n1, bx, maxc);
  const int by_max = std::max(1, std::min(maxc / bx, (n2 + R - 1) / R));
  const int ytiles = (n2 + by_max * R - 1) / (by_max * R);
  const int by = (n2 + ytiles * R - 1) / (ytiles * R);
  const int tile_y = by * R;
  const int ncw = (bx * by + 31) / 32;
  const int rows = tile_y + 2 * MD;
  constexpr int AL = 128 / (int)sizeof(T);
  auto rnd = [&](int e) { return ((e + AL - 1) / AL) * AL; };
  const int stage_elems = rnd(rows * rowlen), vl_elems = rnd(tile_y * n1);
  const size_t stage_bytes = sizeof(T) * (size_t)(stage_elems + vl_elems);
  const size_t budget = 227 * 1024 - 256;
  const int S = (int)std::min<size_t>(8, budget / stage_bytes);
  RS_CHECK(S >= 2, RSDFT_ERR_UNSUPPORTED, "stencil stage (%zu B) does not fit shared memory twice", stage_bytes);
  const int bar_off = (int)(stage_bytes * S);
  const size_t smem = (size_t)bar_off + 16 * (size_t)S + 16;
  int zch = 1;
  double best = -1.0;
  for (int zc = 1; zc <= 8; zc *= 2) {
    const int tz = (n3 + zc - 1) / zc;
    if (zc > 1 && tz < 2 * MD) break;
    const long long items = (long long)ytiles * ((n3 + tz - 1) / tz) * nb;
    const long long grid = std::min<long long>(items, nsm);
    const double bal = (double)items / (double)(grid * ((items + grid - 1) / grid));
    const double score = bal * (double)tz / (tz + 0.25 * 2 * MD);
    if (score > best + 1e-3) {
      best = score;
      zch = zc;
    }
  }
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;
  WsArgs<T, MD> a{};
  a.psi = psi;
  a.out = out;
  a.ld = (long long)ld;
  const bool f32 = std::is_same<T, float>::value;
  a.vloc = (f32 ? (const T*)c.vloc32.as<float>() : (const T*)c.vloc64.as<double>()) + (size_t)s * c.ng;
  a.n1 = n1;
  a.n2 = n2;
  a.n3 = n3;
  a.tile_y = tile_y;
  a.tz = tz;
  a.ytiles = ytiles;
  a.zch = zch;
  a.nb = nb;
  a.bx = bx;
  a.by = by;
  a.ncw = ncw;
  a.stage_elems = stage_elems;
  a.vl_elems = vl_elems;
  a.nst = S;
  a.bar_off = bar_off;
  a.c0 = (T)(c.p.coef_lap0 + c.kp[k].const_k2);
  for (int m = 0; m < MD; ++m) {
    a.cx[m] = (T)c.p.coef_lap[0][m];
    a.cy[m] = (T)c.p.coef_lap[1][m];
    a.cz[m] = (T)c.p.coef_lap[2][m];
    for (int d = 0; d < 3; ++d) a.cs[d][m] = (T)c.kp[k].coef_nabk[d][m];
  }
  a.status = c.d_status;
  a.polls = c.wait_polls >= 0 ? (uint32_t)c.wait_polls : kWaitPolls;
  {  // configuration, readable through rsdft_gpu_profile_get
    const std::string pre = f32 ? "stencil" : "stencil64";
    c.tune_ms[pre + "_stages"] = S;
    c.tune_ms[pre + "_tile_y"] = tile_y;
    c.tune_ms[pre + "_warps"] = ncw + 1;
    c.tune_ms[pre + "_zchunks"] = zch;
    c.tune_ms[pre + "_smem_kb"] = smem / 1024.0;
  }
  const long long nwork = (long long)ytiles * zch * nb;
  const int grid = (int)std::min<long long>(nwork, nsm);
  const double e = (double)sizeof(T);
  ProfScope ps(c, "hpsi_stencil", e * (4.0 * (double)c.ng * nb + (double)c.ng));
  kern<<<grid, (ncw + 1) * 32, smem, c.stream>>>(a);
  c.launches++;
  return check_launch("hpsi_stencil_cplx");
}

template int launch_stencil_ws_c<float, 6>(Ctx&, int, int, const float*, float*, size_t, int);
template int launch_stencil_ws_c<float, 4>(Ctx&, int, int, const float*, float*, size_t, int);
template int launch_stencil_ws_c<double, 6>(Ctx&, int, int, const double*, double*, size_t, int);
template int launch_stencil_ws_c<double, 4>(Ctx&, int, int, const double*, double*, size_t, int);

}  // namespace rsdft
