// Many-band hpsi for the real8 (Gamma) build: H psi = T psi + Vloc psi + V_NL psi.
//
// Reference semantics (restated, not translated):
//   kinetic + Vloc  src/kinetic/d_kinetic_sol_module.f90:244-292  (Md=6 star stencil,
//                   (coef_lap0 + Vloc) on the centre, periodic halo src/bc/bcset_3_module.f90)
//   nonlocal        src/ps_nloc_mr_module.f90:1159-1258 (gather uVunk = dV sum uVk psi(JJP),
//                   Dij pairs, scatter psi(JJP) += uVk * sum Dij uVunk); the KB form
//                   src/d_ps_nloc2_op_module.f90:146-288 is the diagonal-Dij case.
//
// Design (B200): one pass over psi per band.  A CTA owns an (N1 x TY) column of the grid for
// one band and streams it along z.
//  * Each xy-plane of the column (with an Md-deep y halo, periodic rows wrapped) and the
//    matching V_loc tile are staged into shared memory by the bulk-copy (TMA) engine through an
//    S-deep mbarrier ring issued S-1 planes ahead.
//  * Compute warps: x taps wrap inside the staged row (the CTA holds full rows), y taps read
//    neighbouring staged rows, z taps are pushed into 2*Md+1 rotating register accumulators,
//    so every plane is read once from memory; all operands of a step come from shared memory.
//  * Four nonlocal warps run ahead of the compute warps: for each plane they evaluate the
//    projector scatter sum_a sum_p uV_a,p(r) c_b[a,p] from per-(point, atom) records (loads
//    batched several records deep per thread) and the band's coefficient row (staged once in
//    shared memory), accumulate it into a plane buffer and hand it over through a second
//    mbarrier ring.
// The projector gather + Dij runs before, in an atom-centred kernel that writes the
// coefficient rows c_b (atom-major, PG-padded).
#include "stencil.cuh"

namespace rsdft {

// One plane step of the z-push accumulators for rotation slot S (compile-time): add the plane's
// xy part into its own slot, push its z taps into slots S-m and S+m, emit slot S-MD (complete)
// and clear it for reuse.
template <typename T, int MD, int R, int V, int S>
__device__ __forceinline__ void rot_step(T (&acc)[2 * MD + 1][R][V], const T (&v)[R][V], const T (&t)[R][V],
                                         const T (&cz)[MD], bool fin, T* orow, size_t rstride, const bool (&rowok)[R]) {
  constexpr int NQ = 2 * MD + 1;
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < V; ++i) acc[S][r][i] += t[r][i];
#pragma unroll
  for (int m = 1; m <= MD; ++m)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < V; ++i) {
        acc[(S - m + NQ) % NQ][r][i] += cz[m - 1] * v[r][i];
        acc[(S + m) % NQ][r][i] += cz[m - 1] * v[r][i];
      }
  constexpr int FS = (S + NQ - MD) % NQ;
  if (fin) {
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (rowok[r]) stv<T, V>(orow + r * rstride, acc[FS][r]);
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int i = 0; i < V; ++i) acc[FS][r][i] = T(0);
}

template <typename T, int MD, int R, int V, int S>
__device__ __forceinline__ void rot_case(T (&acc)[2 * MD + 1][R][V], const T (&v)[R][V], const T (&t)[R][V],
                                         const T (&cz)[MD], bool fin, T* orow, size_t rstride, const bool (&rowok)[R]) {
  if constexpr (S < 2 * MD + 1) rot_step<T, MD, R, V, S>(acc, v, t, cz, fin, orow, rstride, rowok);
}

// flat switch over the (at most 13) rotation slots; every case is inlined with constant indices
#define RS_ROT_CASE(S_)                                                       \
  case S_:                                                                    \
    rot_case<T, MD, R, V, S_>(acc, v, t, a.cz, fin, orow, (size_t)n1, rowok); \
    break;

template <typename T, int MD, int R, int S, int S2>
__global__ void __launch_bounds__(256, 1) k_stencil_real(const StArgs<T, MD> a) {
  constexpr int V = VecT<T>::V;
  constexpr int NQ = 2 * MD + 1;
  constexpr int NCH = (MD + V - 1) / V;
  extern __shared__ __align__(128) unsigned char smem[];
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const StLayout L = smem_layout<T>(S, S2, a.stage_elems, a.vl_elems, a.nl_elems, a.ldc, a.rec_slots,
                                     a.rec_slot_bytes);
  T* stages = reinterpret_cast<T*>(smem);
  const int sstride = a.stage_elems + a.vl_elems;
  T* nlbuf = reinterpret_cast<T*>(smem + L.nlbuf);
  T* coef_s = reinterpret_cast<T*>(smem + L.coef);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* nlfull = bar + S;
  uint64_t* nlempty = nlfull + S2;
  uint64_t* recfull = nlempty + S2;
  int4* rechdr = reinterpret_cast<int4*>(smem + L.hdr);
  unsigned char* recbuf = smem + L.rec;

  const int tid = threadIdx.x;
  const int nthr_c = a.nthr_c;
  const bool compute = tid < nthr_c;
  const bool active = tid < a.nact;
  const int tx = tid % a.bx, ty = tid / a.bx;
  const int x0 = tx * V;
  const int yl = ty * R;
  const int y0 = blockIdx.x * a.tile_y;
  const int z0 = blockIdx.y * a.tz;
  const int zend = min(z0 + a.tz, n3);
  const int rows = a.tile_y + 2 * MD;
  const int nplanes = (zend - z0) + 2 * MD;
  const int ty_valid = min(a.tile_y, n2 - y0);
  const long long band = blockIdx.z;
  const T* src = a.psi + band * a.ld;
  T* dst = a.out + band * a.ld;
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

  if (!compute) {
    if (nl_on) nl_warps<T, MD, S2>(a, nlbuf, coef_s, nlfull, nlempty, recfull, rechdr, recbuf, tid, nthr_c, z0, zend, y0, ty_valid);
    return;
  }

  // ---------------- compute warps ----------------
  auto issue = [&](int q) {
    const int zg = pmod(z0 - MD + q, n3);
    T* st = stages + (size_t)(q % S) * sstride;
    uint64_t* br = &bar[q % S];
    const int p = z0 - MD + q;
    const bool inch = p >= z0 && p < zend;
    const uint32_t bytes = (uint32_t)((size_t)rows * n1 * sizeof(T)) + (inch ? (uint32_t)((size_t)ty_valid * n1 * sizeof(T)) : 0u);
    mbar_arrive_expect_tx(br, bytes);
    int r = 0;
    while (r < rows) {
      const int gy = pmod(y0 - MD + r, n2);
      const int len = min(rows - r, n2 - gy);
      bulk_g2s(st + (size_t)r * n1, src + ((size_t)zg * n2 + gy) * n1, (uint32_t)((size_t)len * n1 * sizeof(T)), br);
      r += len;
    }
    if (inch)
      bulk_g2s(st + a.stage_elems, a.vloc + ((size_t)p * n2 + y0) * n1, (uint32_t)((size_t)ty_valid * n1 * sizeof(T)), br);
  };
  if (tid == 0)
    for (int q = 0; q < S - 1 && q < nplanes; ++q) issue(q);

  bool rowok[R];
#pragma unroll
  for (int r = 0; r < R; ++r) rowok[r] = active && (yl + r) < ty_valid;

  T acc[NQ][R][V];
#pragma unroll
  for (int q = 0; q < NQ; ++q)
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < V; ++i) acc[q][r][i] = T(0);

  int issued_upto = min(S - 1, nplanes);
  bool aborted = false;
  // The plane loop is rolled; only the accumulator rotation (a few FMAs per slot) is
  // specialised per slot through a switch, which keeps the instruction footprint small.
  for (int q = 0; q < nplanes; ++q) {
    if (tid == 0 && q + S - 1 < nplanes) {
      fence_proxy_async_smem();
      issue(q + S - 1);
      issued_upto = q + S;
    }
    bool ok = mbar_wait_bounded(&bar[q % S], (uint32_t)((q / S) & 1), kWaitPolls);
    const T* pl = stages + (size_t)(q % S) * sstride;
    const int p = z0 - MD + q;
    const bool inch = p >= z0 && p < zend;
    T v[R][V], t[R][V];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int i = 0; i < V; ++i) t[r][i] = T(0);
    if (active) {
#pragma unroll
      for (int r = 0; r < R; ++r) ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + x0, v[r]);
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int i = 0; i < V; ++i) v[r][i] = T(0);
    }
    if (inch) {
      // nonlocal plane buffer for p (filled by the nonlocal warps)
      const int pi = p - z0;
      const int slot = pi % S2;
      const T* nl = nlbuf + (size_t)slot * a.nl_elems;
      if (nl_on) ok = mbar_wait_bounded(&nlfull[slot], (uint32_t)((pi / S2) & 1), kWaitPolls) && ok;
      if (active) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          T vl[V], nv[V];
          if (rowok[r]) {
            ldv<T, V>(pl + a.stage_elems + (size_t)(yl + r) * n1 + x0, vl);
            if (nl_on) {
              ldv<T, V>(nl + (size_t)(yl + r) * n1 + x0, nv);
            } else {
#pragma unroll
              for (int i = 0; i < V; ++i) nv[i] = T(0);
            }
          } else {
#pragma unroll
            for (int i = 0; i < V; ++i) vl[i] = nv[i] = T(0);
          }
#pragma unroll
          for (int i = 0; i < V; ++i) t[r][i] = (a.c0 + vl[i]) * v[r][i] + nv[i];
          // x taps: the full periodic row is staged; chunks wrap modulo N1
          T w[(2 * NCH + 1) * V];
#pragma unroll
          for (int i = 0; i < V; ++i) w[NCH * V + i] = v[r][i];
#pragma unroll
          for (int ch = 1; ch <= NCH; ++ch) {
            T lf[V], rt[V];
            ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + pmod(x0 - ch * V, n1), lf);
            ldv<T, V>(pl + (size_t)(yl + r + MD) * n1 + pmod(x0 + ch * V, n1), rt);
#pragma unroll
            for (int i = 0; i < V; ++i) {
              w[(NCH - ch) * V + i] = lf[i];
              w[(NCH + ch) * V + i] = rt[i];
            }
          }
#pragma unroll
          for (int i = 0; i < V; ++i)
#pragma unroll
            for (int m = 1; m <= MD; ++m) t[r][i] += a.cx[m - 1] * (w[NCH * V + i - m] + w[NCH * V + i + m]);
        }
        // y taps
#pragma unroll
        for (int dy = -MD; dy < R + MD; ++dy) {
          T rv[V];
          if (dy >= 0 && dy < R) {
#pragma unroll
            for (int i = 0; i < V; ++i) rv[i] = v[dy >= 0 && dy < R ? dy : 0][i];
          } else {
            ldv<T, V>(pl + (size_t)(yl + dy + MD) * n1 + x0, rv);
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int m = dy > r ? dy - r : r - dy;
            if (m >= 1 && m <= MD) {
#pragma unroll
              for (int i = 0; i < V; ++i) t[r][i] += a.cy[(m >= 1 ? m : 1) - 1] * rv[i];
            }
          }
        }
      }
      if (nl_on) mbar_arrive(&nlempty[slot]);
    }
    // accumulate plane p (xy part into its own slot, z taps into p-m / p+m) and emit p-MD
    const int zo = p - MD;
    const bool fin = zo >= z0 && zo < zend;
    T* orow = dst + ((size_t)(fin ? zo : 0) * n2 + (y0 + yl)) * n1 + x0;
    switch (q % NQ) {
      RS_ROT_CASE(0) RS_ROT_CASE(1) RS_ROT_CASE(2) RS_ROT_CASE(3) RS_ROT_CASE(4) RS_ROT_CASE(5)
      RS_ROT_CASE(6) RS_ROT_CASE(7) RS_ROT_CASE(8) RS_ROT_CASE(9) RS_ROT_CASE(10) RS_ROT_CASE(11)
      RS_ROT_CASE(12)
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

// ---------------------------------------------------------------------------
// nonlocal gather + Dij (atom-centred):
//   c_b[g*PG + p] = sum_q D_g[p][q] dV sum_j uV_g(j,q) psi_b(JJ_g(j))
// ---------------------------------------------------------------------------
template <typename T, int PG, int BB>
__global__ void __launch_bounds__(256) k_nl_gather_real(const T* __restrict__ psi, long long ld, int nb,
                                                        const int* __restrict__ gofs, const int* __restrict__ gjj,
                                                        const T* __restrict__ gw, const double* __restrict__ gD,
                                                        double dV, T* coef, int ldc) {
  const int g = blockIdx.x;
  const int b0 = blockIdx.y * BB;
  const int f0 = gofs[g], f1 = gofs[g + 1];
  T acc[BB][PG];
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) acc[bb][p] = T(0);
  for (int j = f0 + threadIdx.x; j < f1; j += blockDim.x) {
    const int idx = __ldg(gjj + j);
    T w[PG];
#pragma unroll
    for (int p = 0; p < PG; ++p) w[p] = __ldg(gw + (size_t)j * PG + p);
#pragma unroll
    for (int bb = 0; bb < BB; ++bb) {
      if (b0 + bb < nb) {
        const T v = __ldg(psi + (long long)(b0 + bb) * ld + idx);
#pragma unroll
        for (int p = 0; p < PG; ++p) acc[bb][p] += w[p] * v;
      }
    }
  }
  __shared__ T red[8][BB * PG];
  __shared__ double u[BB * PG];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int bb = 0; bb < BB; ++bb)
#pragma unroll
    for (int p = 0; p < PG; ++p) {
      T x = acc[bb][p];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if (lane == 0) red[wid][bb * PG + p] = x;
    }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (threadIdx.x < BB * PG) {
    double t = 0.0;
    for (int w2 = 0; w2 < nw; ++w2) t += (double)red[w2][threadIdx.x];
    u[threadIdx.x] = t * dV;
  }
  __syncthreads();
  if (threadIdx.x < BB * PG) {
    const int bb = threadIdx.x / PG, p = threadIdx.x % PG;
    if (b0 + bb < nb) {
      double cfs = 0.0;
#pragma unroll
      for (int q = 0; q < PG; ++q) cfs += gD[((size_t)g * PG + p) * PG + q] * u[bb * PG + q];
      coef[(long long)(b0 + bb) * ldc + g * PG + p] = (T)cfs;
    }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
template <typename T, int PG, int BB>
static void launch_gather(Ctx& c, const T* psi, size_t ld, int nb, T* coef, const T* gw) {
  NonlocalTables& nl = c.nl;
  dim3 grid(nl.ngroups, (nb + BB - 1) / BB);
  k_nl_gather_real<T, PG, BB><<<grid, 256, 0, c.stream>>>(psi, (long long)ld, nb, nl.gofs.as<int>(), nl.gjj.as<int>(),
                                                           gw, nl.gD.as<double>(), c.p.dv, coef, nl.ngroups * PG);
  c.launches++;
}

template <typename T>
static int nl_gather(Ctx& c, int k, const T* psi, size_t ld, int nb, T* coef) {
  NonlocalTables& nl = c.nl;
  const T* gw = std::is_same<T, double>::value ? nl.perk[k].gw64.as<T>() : nl.perk[k].gw32.as<T>();
  const double bytes = (double)sizeof(T) * nl.ftotal * ((double)nb + nl.pg) + 4.0 * nl.ftotal;
  ProfScope ps(c, "nl_gather", bytes);
  switch (nl.pg) {
    case 1: launch_gather<T, 1, 8>(c, psi, ld, nb, coef, gw); break;
    case 4: launch_gather<T, 4, 8>(c, psi, ld, nb, coef, gw); break;
    case 9: launch_gather<T, 9, 4>(c, psi, ld, nb, coef, gw); break;
    case 16: launch_gather<T, 16, 2>(c, psi, ld, nb, coef, gw); break;
    default: RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "projectors per atom > 16 not built in");
  }
  return check_launch("nl_gather");
}

// vloc_override / c0_shift: the kinetic-only operator (T + shift) used for training targets
template <typename T, int MD>
static int launch_stencil(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, const T* coef,
                          const T* vloc_override = nullptr, double c0_shift = 0.0) {
  constexpr int V = VecT<T>::V;
  constexpr int R = 2;
  constexpr int S = sizeof(T) == 4 ? 6 : 5;
  constexpr int S2 = 3;
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3;
  RS_CHECK(n1 % V == 0 && n1 / V <= 256, RSDFT_ERR_UNSUPPORTED, "N1=%d must be a multiple of %d (<= %d)", n1, V,
           256 * V);
  RS_CHECK(ld % V == 0, RSDFT_ERR_ARG, "leading dimension must be a multiple of %d", V);
  auto kern = k_stencil_real<T, MD, R, S, S2>;
  static int max_block = 0;  // one per template instantiation: block limit at this register count
  if (!max_block) {
    if constexpr (std::is_same<T, float>::value) {
      RS_TRY((stencil_f32_block_limit<MD, S, S2>(&max_block)));
    } else {
      cudaFuncAttributes fa{};
      RS_CUDA(cudaFuncGetAttributes(&fa, kern));
      max_block = fa.maxThreadsPerBlock;
    }
  }
  const int max_c = ((max_block - 32 * kNLW) / 32) * 32;
  const int bx = n1 / V;
  RS_CHECK(bx <= max_c, RSDFT_ERR_UNSUPPORTED, "N1=%d needs %d threads per row; this build allows %d", n1, bx, max_c);
  int by = std::max(1, std::min(256, max_c) / bx);
  by = std::min(by, (n2 + R - 1) / R);
  while (by > 1 && ((bx * by + 31) / 32) * 32 > max_c) --by;
  const int nthr_c = ((bx * by + 31) / 32) * 32;
  const int tile_y = by * R;
  const int rows = tile_y + 2 * MD;
  const int align_el = 128 / (int)sizeof(T);
  auto rnd = [&](int e) { return ((e + align_el - 1) / align_el) * align_el; };
  const int stage_elems = rnd(rows * n1), vl_elems = rnd(tile_y * n1), nl_elems = rnd(tile_y * n1);
  const bool nl_on = c.nl.nproj > 0 && coef != nullptr;
  const int ldc = nl_on ? c.nl.ngroups * c.nl.pg : 0;
  // record ring: sized for the largest (plane, y-tile) record segment, 3 or 2 slots if they fit
  int rec_slots = 0, rec_cap = 0, rec_cap_rp = 0, rec_slot_bytes = 0;
  if (nl_on) {
    auto it = c.nl.seg_max.find(tile_y);
    if (it == c.nl.seg_max.end()) {
      int mx = 0;
      const std::vector<int>& rp = c.nl.h_rowptr;
      for (int p = 0; p < n3; ++p)
        for (int y0 = 0; y0 < n2; y0 += tile_y) {
          const size_t b0 = ((size_t)p * n2 + y0) * n1, b1 = b0 + (size_t)std::min(tile_y, n2 - y0) * n1;
          mx = std::max(mx, rp[b1] - rp[b0]);
        }
      it = c.nl.seg_max.emplace(tile_y, mx).first;
    }
    rec_cap = ((it->second + 6) + 3) / 4 * 4;
    rec_cap_rp = ((tile_y * n1 + 1 + 6) + 3) / 4 * 4;
    rec_slot_bytes =
        (int)(((size_t)rec_cap_rp * 4 + (size_t)rec_cap * (4 + c.nl.pg * sizeof(T)) + 127) / 128 * 128);
    for (int rs = kRecSlotsMax; rs >= 2; --rs)
      if (smem_layout<T>(S, S2, stage_elems, vl_elems, nl_elems, ldc, rs, rec_slot_bytes).total <= 225 * 1024) {
        rec_slots = rs;
        break;
      }
  }
  const size_t smem = smem_layout<T>(S, S2, stage_elems, vl_elems, nl_elems, ldc, rec_slots, rec_slot_bytes).total;
  RS_CHECK(smem <= 225 * 1024, RSDFT_ERR_UNSUPPORTED, "stencil stages (%zu B) exceed shared memory", smem);
  const int ytiles = (n2 + tile_y - 1) / tile_y;
  int zch = 1;
  while ((long long)ytiles * zch * nb < 4 * 148 && n3 / (zch * 2) >= 16) zch *= 2;
  const int tz = (n3 + zch - 1) / zch;
  zch = (n3 + tz - 1) / tz;

  StArgs<T, MD> a;
  a.psi = psi;
  a.out = out;
  a.ld = (long long)ld;
  a.vloc = vloc_override ? vloc_override
                         : (std::is_same<T, double>::value ? c.vloc64.as<T>() : c.vloc32.as<T>()) + (size_t)s * c.ng;
  a.n1 = n1; a.n2 = n2; a.n3 = n3;
  a.tile_y = tile_y; a.tz = tz;
  a.bx = bx; a.nact = bx * by; a.nthr_c = nthr_c;
  a.stage_elems = stage_elems; a.vl_elems = vl_elems; a.nl_elems = nl_elems;
  a.c0 = (T)(c.p.coef_lap0 + c.kp[k].const_k2 + c0_shift);
  for (int m = 0; m < MD; ++m) {
    a.cx[m] = (T)c.p.coef_lap[0][m];
    a.cy[m] = (T)c.p.coef_lap[1][m];
    a.cz[m] = (T)c.p.coef_lap[2][m];
  }
  a.rec_rowptr = nl_on ? c.nl.rec_rowptr.as<int>() : nullptr;
  a.rec_pt = nl_on ? c.nl.rec_pt.as<int>() : nullptr;
  a.rec_g = nl_on ? c.nl.rec_g.as<int>() : nullptr;
  a.rec_u = nl_on ? (std::is_same<T, double>::value ? c.nl.perk[k].ru64.as<T>() : c.nl.perk[k].ru32.as<T>()) : nullptr;
  a.pg = c.nl.pg;
  a.coef = coef;
  a.ldc = ldc;
  a.status = c.d_status;
  a.rec_slots = rec_slots;
  a.rec_cap = rec_cap;
  a.rec_cap_rp = rec_cap_rp;
  a.rec_slot_bytes = rec_slot_bytes;
  static bool attr_done = false;  // one per template instantiation
  if (!attr_done && !std::is_same<T, float>::value) {
    RS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 225 * 1024));
    attr_done = true;
  }
  dim3 grid(ytiles, zch, nb), block(nthr_c + 32 * kNLW);
  // algorithmic bytes: read psi + write H psi per band, V_loc and the projector records once
  const double alg_bytes = (double)sizeof(T) * (2.0 * (double)c.ng * nb + (double)c.ng) +
                           (nl_on ? 4.0 * (double)(c.ng + 1) + (8.0 + sizeof(T) * c.nl.pg) * c.nl.ftotal : 0.0);
  ProfScope ps(c, "hpsi_stencil", alg_bytes);
  if constexpr (std::is_same<T, float>::value) {
    RS_TRY((launch_stencil_f32<MD, S, S2>(a, grid, block, smem, c.stream)));
  } else {
    kern<<<grid, block, smem, c.stream>>>(a);
  }
  c.launches++;
  return check_launch("hpsi_stencil");
}

template <typename T>
int hpsi_real(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "real hpsi called on a complex16 context");
  RS_CHECK(c.kp[k].set || c.p.nk == 1, RSDFT_ERR_STATE, "k-point %d not set", k + 1);
  RS_CHECK(c.vloc_set[s], RSDFT_ERR_STATE, "Vloc for spin %d not set", s + 1);
  if (nb <= 0) return 0;
  T* coef = nullptr;
  if (c.nl.nproj > 0) {
    RS_TRY(nl_prepare_k(c, k));
    RS_TRY(c.ws_coef.ensure((size_t)nb * c.nl.ngroups * c.nl.pg * sizeof(T)));
    coef = c.ws_coef.as<T>();
    RS_TRY(nl_gather<T>(c, k, psi, ld, nb, coef));
  }
  if (c.p.md == 6) return launch_stencil<T, 6>(c, k, s, psi, out, ld, nb, coef);
  if (c.p.md == 4) return launch_stencil<T, 4>(c, k, s, psi, out, ld, nb, coef);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}

template int hpsi_real<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_real<double>(Ctx&, int, int, const double*, double*, size_t, int);

// hpsi with caller-provided scratch for the nonlocal coefficient rows (coef_cap elements of
// T); performs no device allocation.
template <typename T>
int hpsi_real_scratch(Ctx& c, int k, int s, const T* psi, T* out, size_t ld, int nb, T* coef, size_t coef_cap) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "real hpsi called on a complex16 context");
  RS_CHECK(c.kp[k].set || c.p.nk == 1, RSDFT_ERR_STATE, "k-point %d not set", k + 1);
  RS_CHECK(c.vloc_set[s], RSDFT_ERR_STATE, "Vloc for spin %d not set", s + 1);
  if (nb <= 0) return 0;
  T* cf = nullptr;
  if (c.nl.nproj > 0) {
    RS_TRY(nl_prepare_k(c, k));
    const size_t need = (size_t)nb * c.nl.ngroups * c.nl.pg;
    RS_CHECK(coef != nullptr && need <= coef_cap, RSDFT_ERR_ARG,
             "nonlocal scratch too small: %zu coefficients needed, %zu available", need, coef_cap);
    cf = coef;
    RS_TRY(nl_gather<T>(c, k, psi, ld, nb, cf));
  }
  if (c.p.md == 6) return launch_stencil<T, 6>(c, k, s, psi, out, ld, nb, cf);
  if (c.p.md == 4) return launch_stencil<T, 4>(c, k, s, psi, out, ld, nb, cf);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}
template int hpsi_real_scratch<double>(Ctx&, int, int, const double*, double*, size_t, int, double*, size_t);

// y = (T + shift) x with T the finite-difference kinetic operator alone (no V_loc, no
// projectors), real Gamma build, FP32.
int kinetic_shifted(Ctx& c, const float* x, float* y, size_t ld, int nb, double shift) {
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "kinetic_shifted: real build only");
  if (nb <= 0) return 0;
  if (!c.vzero.p || c.vzero.bytes < sizeof(float) * c.ng) {
    RS_TRY(c.vzero.ensure(sizeof(float) * c.ng));
    RS_CUDA(cudaMemsetAsync(c.vzero.p, 0, sizeof(float) * c.ng, c.stream));
  }
  const float* vz = c.vzero.as<float>();
  if (c.p.md == 6) return launch_stencil<float, 6>(c, 0, 0, x, y, ld, nb, nullptr, vz, shift);
  if (c.p.md == 4) return launch_stencil<float, 4>(c, 0, 0, x, y, ld, nb, nullptr, vz, shift);
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "Md=%d not built in (4 and 6 are)", c.p.md);
}

}  // namespace rsdft
