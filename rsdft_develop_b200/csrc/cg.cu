// Batched band-by-band preconditioned CG and the hprsdft preconditioner, real8 and complex16.
//
// Reference: d_/z_conjugate_gradient_1 (src/conjugate_gradient/cg_module.f90:112-431 and
// :434-754) with MB_d = 1: every band runs its own CG independently, so all bands of a block
// are advanced together here with per-band state (E, E1, rb, gkgk, res, active flag) kept on
// the device.  A band that leaves the reference's icg loop early (|E-E1| < 1e-15, which
// follows a rejected step, :233) is masked out for the rest of the call, which reproduces the
// per-band exits of MB_d = 1 exactly.  precond_hprsdft
// (src/conjugate_gradient/cgpc_hprsdft_module.f90:133-270) is batched the same way: FP64 bands
// run its CG recurrence (26 passes at mloop = 3), FP32 bands the same mloop steps in s-step
// form (k_pcs_*: Krylov basis, moments, FP64 recurrence on coefficients; 12 passes).
//
// complex16 arrays are handled through their interleaved real view (2*ML0 reals per band,
// the same view the reference's dot_product takes with mm = 2*ML0, cg_module.f90:478):
// every kernel whose coefficients are real works unchanged on that view; only the two
// complex overlaps <p|psi>, <p|H psi>, the 2x2 Hermitian solve (zhegv) and the updates with
// complex coefficients have NC = 2 variants.
//
// Reductions are deterministic: each CTA writes a per-band partial sum and the scalar
// kernels add the partials of a band in a fixed order.  In the real build H x of every band is
// kept in one array (ctx ws_hpsi) so that the fused Gram-Schmidt / subspace step of the sweep
// can take it instead of recomputing it.
#include <cstring>

#include "cgk.cuh"

namespace rsdft {

// 16 bytes of T (4 FP32 or 2 FP64 reals): the unit every CG and preconditioner thread loads and
// stores, so that each memory instruction moves 16 bytes.
template <typename T>
struct Vec {
  static constexpr int W = 16 / (int)sizeof(T);
  T v[W];
};
template <typename T>
__device__ __forceinline__ Vec<T> ldv(const T* p) {
  Vec<T> r;
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
  } else {
    const double2 a = *reinterpret_cast<const double2*>(p);
    r.v[0] = a.x; r.v[1] = a.y;
  }
  return r;
}
template <typename T>
__device__ __forceinline__ void stv(T* p, const Vec<T>& r) {
  if constexpr (sizeof(T) == 4)
    *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
  else
    *reinterpret_cast<double2*>(p) = make_double2(r.v[0], r.v[1]);
}

// NC = 2 loops run over complex points (pairs of reals)
#define BAND_LOOP(k, NC)                                                    \
  const int b = blockIdx.y;                                                 \
  const size_t off = (size_t)b * (k).ng;                                    \
  const size_t npt = (k).ng / (NC);                                         \
  const size_t per = (npt + (k).nch - 1) / (k).nch;                         \
  const size_t i0 = per * blockIdx.x, i1 = min(npt, i0 + per);

// Elementwise walk of a band in 16-byte groups of VW reals (complex bands: VW / 2 points per
// group); the band's groups are split into k.nch contiguous chunks, one per CTA.  Bands hold a
// multiple of VW reals (the stencils require N1 to be a multiple of VW).
#define GROUP_LOOP(k, T)                                                    \
  constexpr int VW = Vec<T>::W;                                             \
  const int b = blockIdx.y;                                                 \
  const size_t off = (size_t)b * (k).ng;                                    \
  const size_t ngr = (k).ng / VW;                                           \
  const size_t per = (ngr + (k).nch - 1) / (k).nch;                         \
  const size_t g0 = per * blockIdx.x, g1 = min(ngr, g0 + per);

// ---------------------------------------------------------------------------
// elementwise + reduction kernels on the real view, 16-byte accesses
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_dot(Blk k, const T* __restrict__ a, const T* __restrict__ bb,
                                                  int act_idx) {
  GROUP_LOOP(k, T);
  if (act_idx >= 0 && SC(k, act_idx, b) == 0.0) return;
  double v[1] = {0.0};
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> x = ldv(a + e), y = ldv(bb + e);
#pragma unroll
    for (int i = 0; i < VW; ++i) v[0] += (double)x.v[i] * (double)y.v[i];
  }
  block_partials<1>(v, k, b);
}

// g = gfac (hx - E x); partial |g|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_make_g(Blk k, const T* __restrict__ x, const T* __restrict__ hx,
                                                     T* __restrict__ g, double gfac) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  const double E = SC(k, S_E, b);
  double v[1] = {0.0};
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> xv = ldv(x + e), hv = ldv(hx + e);
    Vec<T> gv;
#pragma unroll
    for (int i = 0; i < VW; ++i) {
      gv.v[i] = (T)(gfac * ((double)hv.v[i] - E * (double)xv.v[i]));
      v[0] += (double)gv.v[i] * (double)gv.v[i];
    }
    stv(g + e, gv);
  }
  block_partials<1>(v, k, b);
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_copy(Blk k, const T* __restrict__ src, T* __restrict__ dst) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) stv(dst + off + gi * VW, ldv(src + off + gi * VW));
}

// p = Pg + beta p
template <typename T>
__global__ void __launch_bounds__(kThreads) k_make_p(Blk k, const T* __restrict__ pg, T* __restrict__ p, int first) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  const T beta = (T)SC(k, S_BETA, b);
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    Vec<T> pv = ldv(pg + e);
    if (!first) {
      const Vec<T> po = ldv(p + e);
#pragma unroll
      for (int i = 0; i < VW; ++i) pv.v[i] = pv.v[i] + beta * po.v[i];
    }
    stv(p + e, pv);
  }
}

// the six dot products of the line minimisation (cg_module.f90:288-296, :623-630);
// NC = 1 adds <hx|hx>, <hx|hp>, <hp|hp>, <x|hp> for the estimate of |g|^2 after the step (the
// reject test ahead of the fused x update); NC = 2 adds Im<p|x> and Im<p|hx> in slots 6 and 7
template <typename T, int NC>
__global__ void __launch_bounds__(kThreads) k_dots6(Blk k, const T* __restrict__ x, const T* __restrict__ p,
                                                    const T* __restrict__ hx, const T* __restrict__ hp) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  constexpr int ND = NC == 1 ? 10 : 8;
  double v[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) v[d] = 0.0;
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> xv = ldv(x + e), pv = ldv(p + e), hv = ldv(hx + e), qv = ldv(hp + e);
    if constexpr (NC == 1) {
#pragma unroll
      for (int i = 0; i < VW; ++i) {
        const double xi = xv.v[i], pi = pv.v[i], hxi = hv.v[i], hpi = qv.v[i];
        v[0] += xi * xi;
        v[1] += pi * xi;
        v[2] += pi * pi;
        v[3] += xi * hxi;
        v[4] += pi * hxi;
        v[5] += pi * hpi;
        v[6 % ND] += hxi * hxi;
        v[7 % ND] += hxi * hpi;
        v[8 % ND] += hpi * hpi;
        v[9 % ND] += xi * hpi;
      }
    } else {
#pragma unroll
      for (int j = 0; j < VW / 2; ++j) {
        const double xr = xv.v[2 * j], xm = xv.v[2 * j + 1], pr = pv.v[2 * j], pm = pv.v[2 * j + 1];
        const double hr = hv.v[2 * j], hm = hv.v[2 * j + 1], qr = qv.v[2 * j], qm = qv.v[2 * j + 1];
        v[0] += xr * xr + xm * xm;
        v[1] += pr * xr + pm * xm;
        v[2] += pr * pr + pm * pm;
        v[3] += xr * hr + xm * hm;
        v[4] += pr * hr + pm * hm;
        v[5] += pr * qr + pm * qm;
        v[ND - 2] += pr * xm - pm * xr;
        v[ND - 1] += pr * hm - pm * hr;
      }
    }
  }
  block_partials<ND>(v, k, b);
}

// hx = u1 hx + u2 hp ; g = gfac (hx - W (u1 x + u2 p)) ; partial |g|^2.  Real build: also
// x = u1 x + u2 p in the same pass for bands whose update k_sc_solve2 did not defer (S_DEF = 0).
template <typename T, int NC>
__global__ void __launch_bounds__(kThreads) k_update_hg(Blk k, T* __restrict__ x, const T* __restrict__ p,
                                                        T* __restrict__ hx, const T* __restrict__ hp,
                                                        T* __restrict__ g, double gfac) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  const double u1 = SC(k, S_U1, b), u2 = SC(k, S_U2, b), W = SC(k, S_W, b);
  const double u1i = SC(k, S_U1I, b), u2i = SC(k, S_U2I, b);
  const bool upx = NC == 1 && SC(k, S_DEF, b) == 0.0;
  double v[1] = {0.0};
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> hv = ldv(hx + e), qv = ldv(hp + e), xv = ldv(x + e), pv = ldv(p + e);
    Vec<T> nh, gv, xn;
    if constexpr (NC == 1) {
#pragma unroll
      for (int i = 0; i < VW; ++i) {
        const T ht = (T)(u1 * (double)hv.v[i] + u2 * (double)qv.v[i]);
        nh.v[i] = ht;
        const double xnd = u1 * (double)xv.v[i] + u2 * (double)pv.v[i];
        xn.v[i] = (T)xnd;
        gv.v[i] = (T)(gfac * ((double)ht - W * xnd));
        v[0] += (double)gv.v[i] * (double)gv.v[i];
      }
    } else {
#pragma unroll
      for (int j = 0; j < VW / 2; ++j) {
        const double hr = hv.v[2 * j], hm = hv.v[2 * j + 1], qr = qv.v[2 * j], qm = qv.v[2 * j + 1];
        const T nr = (T)(u1 * hr - u1i * hm + u2 * qr - u2i * qm);
        const T nm = (T)(u1 * hm + u1i * hr + u2 * qm + u2i * qr);
        nh.v[2 * j] = nr;
        nh.v[2 * j + 1] = nm;
        const double xr = xv.v[2 * j], xm = xv.v[2 * j + 1], pr = pv.v[2 * j], pm = pv.v[2 * j + 1];
        const double yr = u1 * xr - u1i * xm + u2 * pr - u2i * pm;
        const double ym = u1 * xm + u1i * xr + u2 * pm + u2i * pr;
        gv.v[2 * j] = (T)(gfac * ((double)nr - W * yr));
        gv.v[2 * j + 1] = (T)(gfac * ((double)nm - W * ym));
        v[0] += (double)gv.v[2 * j] * (double)gv.v[2 * j] + (double)gv.v[2 * j + 1] * (double)gv.v[2 * j + 1];
      }
    }
    stv(hx + e, nh);
    stv(g + e, gv);
    if (upx) stv(x + e, xn);
  }
  block_partials<1>(v, k, b);
}

// x = u1 x + u2 p for accepted bands (complex build; real build: the bands whose update was
// deferred).  Real build, a band k_sc_reject turned down although the estimate let the x update
// go ahead with H x: x = (x - u2 p) / u1 restores the band up to rounding.
template <typename T, int NC>
__global__ void __launch_bounds__(kThreads) k_update_x(Blk k, T* __restrict__ x, const T* __restrict__ p) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  const bool acc = SC(k, S_ACC, b) != 0.0;
  const double u1 = SC(k, S_U1, b), u2 = SC(k, S_U2, b);
  const double u1i = SC(k, S_U1I, b), u2i = SC(k, S_U2I, b);
  if constexpr (NC == 1) {
    const bool def = SC(k, S_DEF, b) != 0.0;
    const bool undo = !acc && !def;
    if (!(acc && def) && !undo) return;
    for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
      const size_t e = off + gi * VW;
      Vec<T> xv = ldv(x + e);
      const Vec<T> pv = ldv(p + e);
#pragma unroll
      for (int i = 0; i < VW; ++i)
        xv.v[i] = undo ? (T)(((double)xv.v[i] - u2 * (double)pv.v[i]) / u1)
                       : (T)(u1 * (double)xv.v[i] + u2 * (double)pv.v[i]);
      stv(x + e, xv);
    }
    return;
  }
  if (!acc) return;
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    Vec<T> xv = ldv(x + e);
    const Vec<T> pv = ldv(p + e);
#pragma unroll
    for (int j = 0; j < VW / 2; ++j) {
      const double xr = xv.v[2 * j], xm = xv.v[2 * j + 1], pr = pv.v[2 * j], pm = pv.v[2 * j + 1];
      xv.v[2 * j] = (T)(u1 * xr - u1i * xm + u2 * pr - u2i * pm);
      xv.v[2 * j + 1] = (T)(u1 * xm + u1i * xr + u2 * pm + u2i * pr);
    }
    stv(x + e, xv);
  }
}

// ---------------------------------------------------------------------------
// per-band scalar kernels (one thread per band)
// ---------------------------------------------------------------------------
__global__ void k_sc_init(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  SC(k, S_E, b) = sum_part(k, b, 0) * dV;
  SC(k, S_E1, b) = 1.0e10;
  SC(k, S_ACT, b) = 1.0;
  SC(k, S_RES, b) = 0.0;
}

__global__ void k_sc_rb(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  SC(k, S_RB, b) = sum_part(k, b, 0) * dV;
}

// loop head: res = rb / c1^2, exit tests (cg_module.f90:231-237, :556-562)
__global__ void k_sc_top(Blk k, double c1sq) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = SC(k, S_RB, b);
  SC(k, S_RES, b) = rb / c1sq;
  if (rb < 0.0 || fabs(SC(k, S_E, b) - SC(k, S_E1, b)) < 1.0e-15) SC(k, S_ACT, b) = 0.0;
}

// rb = <Pg|g> dV ; beta = rb / gkgk ; gkgk = rb
__global__ void k_sc_beta(Blk k, double dV, int first) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = sum_part(k, b, 0) * dV;
  SC(k, S_RB, b) = rb;
  SC(k, S_BETA, b) = first ? 0.0 : rb / SC(k, S_GKGK, b);
  SC(k, S_GKGK, b) = rb;
}

// 2x2 generalised Hermitian eigenproblem A z = w B z (dsygv/zhegv itype 1, cg_module.f90:316,
// :651) by Cholesky B = U^H U and C = U^-H A U^-1, root selection (:317-321) and phase fix
// (real: :322-327, complex: :657-662).  B12 = <psi|p>, A12 = <psi|H p> = conj(<p|H psi>).
template <int NC>
__global__ void k_sc_solve2(Blk k, double dV) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double B11 = sum_part(k, b, 0) * dV, B22 = sum_part(k, b, 2) * dV;
  const double A11 = sum_part(k, b, 3) * dV, A22 = sum_part(k, b, 5) * dV;
  const double B12r = sum_part(k, b, 1) * dV, A12r = sum_part(k, b, 4) * dV;
  const double B12i = NC == 2 ? -sum_part(k, b, 6) * dV : 0.0;
  const double A12i = NC == 2 ? -sum_part(k, b, 7) * dV : 0.0;
  const double E = SC(k, S_E, b);
  bool ok = B11 > 0.0;
  double u11 = 0, u12r = 0, u12i = 0, u22 = 0;
  if (ok) {
    u11 = sqrt(B11);
    u12r = B12r / u11;
    u12i = B12i / u11;
    const double t = B22 - (u12r * u12r + u12i * u12i);
    ok = t > 0.0;
    if (ok) u22 = sqrt(t);
  }
  if (!ok) {  // B not positive definite: keep the band unchanged
    SC(k, S_U1, b) = 1.0;
    SC(k, S_U1I, b) = 0.0;
    SC(k, S_U2, b) = 0.0;
    SC(k, S_U2I, b) = 0.0;
    SC(k, S_W, b) = E;
    SC(k, S_E1, b) = E;
    SC(k, S_DEF, b) = 1.0;
    return;
  }
  // L = U^-H: l11 = 1/u11, l21 = -conj(u12)/(u11 u22), l22 = 1/u22 ; C = L A L^H
  const double l11 = 1.0 / u11, l22 = 1.0 / u22;
  const double l21r = -u12r / (u11 * u22), l21i = u12i / (u11 * u22);
  const double ca = l11 * l11 * A11;
  // C12 = l11 (A11 conj(l21) + A12 l22)
  const double c12r = l11 * (A11 * l21r + A12r * l22);
  const double c12i = l11 * (-A11 * l21i + A12i * l22);
  // C22 = |l21|^2 A11 + 2 l22 Re(l21 A12) + l22^2 A22
  const double cd = (l21r * l21r + l21i * l21i) * A11 + 2.0 * l22 * (l21r * A12r - l21i * A12i) + l22 * l22 * A22;
  const double mean = 0.5 * (ca + cd), r = sqrt(0.25 * (ca - cd) * (ca - cd) + c12r * c12r + c12i * c12i);
  const double w1 = mean - r, w2 = mean + r;
  // eigenvector of w1: (c12, w1 - ca) or (cd - w1, -conj(c12)), the longer one
  double v1r, v1i, v2r, v2i;
  if (r == 0.0) {
    v1r = 1.0; v1i = 0.0; v2r = 0.0; v2i = 0.0;
  } else if (cd - w1 >= ca - w1) {
    v1r = cd - w1; v1i = 0.0; v2r = -c12r; v2i = c12i;
  } else {
    v1r = c12r; v1i = c12i; v2r = w1 - ca; v2i = 0.0;
  }
  const double nv = sqrt(v1r * v1r + v1i * v1i + v2r * v2r + v2i * v2i);
  v1r /= nv; v1i /= nv; v2r /= nv; v2i /= nv;
  // eigenvector of w2: (-conj(v2), conj(v1))
  const double s1r = -v2r, s1i = v2i, s2r = v1r, s2i = -v1i;
  // back-transform z = U^-1 v: z1 = v1/u11 - u12 v2/(u11 u22), z2 = v2/u22
  auto back = [&](double a1r, double a1i, double a2r, double a2i, double& z1r, double& z1i, double& z2r,
                  double& z2i) {
    const double f = 1.0 / (u11 * u22);
    z1r = a1r / u11 - f * (u12r * a2r - u12i * a2i);
    z1i = a1i / u11 - f * (u12r * a2i + u12i * a2r);
    z2r = a2r / u22;
    z2i = a2i / u22;
  };
  double z1r, z1i, z2r, z2i, W = w1;
  back(v1r, v1i, v2r, v2i, z1r, z1i, z2r, z2i);
  if (fabs(w1 - E) > 1.0e-1 && fabs(w2 - E) <= 1.0e-1) {
    W = w2;
    back(s1r, s1i, s2r, s2i, z1r, z1i, z2r, z2i);
  }
  if (NC == 1) {
    if (z1r < 0.0) { z1r = -z1r; z2r = -z2r; }
    z1i = z2i = 0.0;
  } else {
    // multiply by conj(z1)/|z1| so that z1 is real and positive
    const double az = sqrt(z1r * z1r + z1i * z1i);
    const double pr = z1r / az, pi = -z1i / az;
    const double t2r = z2r * pr - z2i * pi, t2i = z2r * pi + z2i * pr;
    z1r = az; z1i = 0.0; z2r = t2r; z2i = t2i;
  }
  SC(k, S_U1, b) = z1r;
  SC(k, S_U1I, b) = z1i;
  SC(k, S_U2, b) = z2r;
  SC(k, S_U2I, b) = z2i;
  SC(k, S_W, b) = W;
  SC(k, S_E1, b) = E;
  SC(k, S_E, b) = W;
  if (NC == 1) {
    // |g'|^2 dV after the step, g' = -2 (u1 (hx - W x) + u2 (hp - W p)), from the dots: the x
    // update may go with the H x / g pass unless the reject test (rb / res > 1e8, k_sc_reject) could
    // turn the step down; within a factor 1e4 of that test it waits for the exact |g'|^2.
    const double xx = B11 / dV, px = B12r / dV, pp = B22 / dV, xh = A11 / dV, ph = A12r / dV, pq = A22 / dV;
    const double hh = sum_part(k, b, 6), hq = sum_part(k, b, 7), qq = sum_part(k, b, 8), xq = sum_part(k, b, 9);
    const double e11 = hh - 2.0 * W * xh + W * W * xx;
    const double e12 = hq - W * xq - W * ph + W * W * px;
    const double e22 = qq - 2.0 * W * pq + W * W * pp;
    const double est = 4.0 * dV * (z1r * z1r * e11 + 2.0 * z1r * z2r * e12 + z2r * z2r * e22);
    SC(k, S_DEF, b) = (est > 1.0e4 * SC(k, S_RES, b) || !(est == est)) ? 1.0 : 0.0;
  }
}

// residual growth guard (cg_module.f90:360-363)
__global__ void k_sc_reject(Blk k, double dV, int* rejected) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  const double rb = sum_part(k, b, 0) * dV;
  SC(k, S_RB, b) = rb;
  if (rb / SC(k, S_RES, b) > 1.0e8) {
    SC(k, S_E, b) = SC(k, S_E1, b);
    SC(k, S_ACC, b) = 0.0;
    atomicAdd(rejected, 1);  // x keeps its value while H x has moved on
  } else {
    SC(k, S_ACC, b) = 1.0;
  }
}

// ---------------------------------------------------------------------------
// preconditioner: 7-point operator A = (c0 - E0) I + sum_d c_d (shift_+ + shift_-), E0 = 0,
// applied to each component of the real view (real coefficients)
// ---------------------------------------------------------------------------
struct PcCoef {
  double c0, c1, c2, c3;
  int n1, n2, n3, nc;
};

// Walk of the CTA's chunk of x-rows (rows of n1 * NCP reals) in groups of W consecutive reals,
// consecutive threads on consecutive groups; per group the periodic neighbour offsets of its
// row (y, z) and the offsets xl / xr, from the group start, of the reals just left and right
// of the group (x, wrapping within the row).  Needs n1 * NCP to be a multiple of W.
#define PC_GROUPS_BEGIN(k, q, T)                                                                 \
  constexpr int VW = Vec<T>::W;                                                                  \
  const int b = blockIdx.y;                                                                      \
  const size_t off = (size_t)b * (k).ng;                                                         \
  const int L = (q).n1 * NCP;                                                                    \
  const int NGR = L / VW;                                                                          \
  const int nrow = (q).n2 * (q).n3;                                                              \
  const int per = (nrow + (k).nch - 1) / (k).nch;                                                \
  const int r0 = per * blockIdx.x, r1 = min(nrow, r0 + per);                                     \
  const long long pln = (long long)(q).n2 * L;                                                   \
  /* (row, group) of the thread's first item, then advanced by kThreads items per step without \
     division: the step is srow rows and sg groups */                                            \
  const int srow = kThreads / NGR, sg = kThreads - srow * NGR;                                  \
  int row = r0 + (int)threadIdx.x / NGR, gq = (int)threadIdx.x - ((int)threadIdx.x / NGR) * NGR;  \
  const int pc_n2 = (q).n2;                                                                      \
  int i2 = row % pc_n2, i3 = row / pc_n2;                                                        \
  for (; row < r1; ) {                                                                           \
    const long long ym = i2 == 0 ? (long long)((q).n2 - 1) * L : -(long long)L;                  \
    const long long yp = i2 == (q).n2 - 1 ? -(long long)((q).n2 - 1) * L : (long long)L;         \
    const long long zm = i3 == 0 ? (long long)((q).n3 - 1) * pln : -pln;                         \
    const long long zp = i3 == (q).n3 - 1 ? -(long long)((q).n3 - 1) * pln : pln;                \
    const long long j = (long long)row * L + (long long)gq * VW;                                  \
    const int xl = gq == 0 ? L - NCP : -NCP;                                                     \
    const int xr = gq == NGR - 1 ? VW - L : VW;
#define PC_GROUPS_END                                                                            \
    gq += sg;                                                                                    \
    int dr = srow;                                                                               \
    if (gq >= NGR) {                                                                             \
      gq -= NGR;                                                                                 \
      ++dr;                                                                                      \
    }                                                                                            \
    row += dr;                                                                                   \
    i2 += dr;                                                                                    \
    while (i2 >= pc_n2) {                                                                        \
      i2 -= pc_n2;                                                                               \
      ++i3;                                                                                      \
    }                                                                                            \
  }

// 7-point operator on the group at j, in the storage type's arithmetic (FP32 bands: FP32 math,
// no per-element conversions); c receives the group's own values.  Same expression per real as
// the scalar form c0 g + c1 (g[x+1] + g[x-1]) + c2 (g[y+1] + g[y-1]) + c3 (g[z+1] + g[z-1]).
template <typename T, int NCP>
__device__ __forceinline__ Vec<T> apply7v(const T* __restrict__ g, long long j, int xl, int xr, long long ym,
                                          long long yp, long long zm, long long zp, const PcCoef& q, Vec<T>& c) {
  constexpr int W = Vec<T>::W;
  c = ldv(g + j);
  const Vec<T> a = ldv(g + j + ym), bq = ldv(g + j + yp), d = ldv(g + j + zm), e = ldv(g + j + zp);
  T lft[NCP], rgt[NCP];
#pragma unroll
  for (int i = 0; i < NCP; ++i) {
    lft[i] = g[j + xl + i];
    rgt[i] = g[j + xr + i];
  }
  Vec<T> o;
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const T xm = i >= NCP ? c.v[i >= NCP ? i - NCP : 0] : lft[i < NCP ? i : 0];
    const T xp = i + NCP < W ? c.v[i + NCP < W ? i + NCP : 0] : rgt[i + NCP >= W ? i + NCP - W : 0];
    o.v[i] = (T)q.c0 * c.v[i] + (T)q.c1 * (xp + xm) + (T)q.c2 * (bq.v[i] + a.v[i]) + (T)q.c3 * (e.v[i] + d.v[i]);
  }
  return o;
}

// R = G - A G (the initial residual for the starting guess PG = G, also the first direction);
// partial |R|^2.  NU (s-step form): also <R|G> and <R|B G>, B G = (A G - c0 G) / c0, the first
// two of nu_i = <B^i R|G> (the later ones follow from the moments, see k_pcs_beta)
template <typename T, int NCP, bool NU = false>
__global__ void __launch_bounds__(kThreads) k_pc_first(Blk k, PcCoef q, const T* __restrict__ G,
                                                       T* __restrict__ R) {
  if (SC(k, S_ACT, blockIdx.y) == 0.0) return;
  T vt = T(0), n0 = T(0), n1 = T(0);  // per-thread partials in the storage type, added in FP64 across threads
  const T c0 = (T)q.c0, ic0 = (T)(1.0 / q.c0);
  {
    PC_GROUPS_BEGIN(k, q, T)
    Vec<T> c;
    const Vec<T> ag = apply7v<T, NCP>(G + off, j, xl, xr, ym, yp, zm, zp, q, c);
    Vec<T> r;
#pragma unroll
    for (int i = 0; i < VW; ++i) {
      r.v[i] = c.v[i] - ag.v[i];
      vt += r.v[i] * r.v[i];
      if (NU) {
        n0 += r.v[i] * c.v[i];
        n1 += r.v[i] * ((ag.v[i] - c0 * c.v[i]) * ic0);
      }
    }
    stv(R + off + j, r);
    PC_GROUPS_END
  }
  if (NU) {
    double v[3] = {(double)vt, (double)n0, (double)n1};
    block_partials<3>(v, k, blockIdx.y);
  } else {
    double v[1] = {(double)vt};
    block_partials<1>(v, k, blockIdx.y);
  }
}

// Qn = R + b Q and F = A Qn = A R + b A Q in one pass (Qn written to a third buffer, since
// the stencil reads Q's neighbours); partial <Qn|F>
template <typename T, int NCP>
__global__ void __launch_bounds__(kThreads) k_pc_dirapply(Blk k, PcCoef q, const T* __restrict__ R,
                                                          const T* __restrict__ Q, T* __restrict__ Qn,
                                                          T* __restrict__ F) {
  if (SC(k, S_PCACT, blockIdx.y) == 0.0) return;
  const T bb = (T)SC(k, S_PCB, blockIdx.y);
  T vt = T(0);
  {
    PC_GROUPS_BEGIN(k, q, T)
    Vec<T> cr, cq;
    const Vec<T> ar = apply7v<T, NCP>(R + off, j, xl, xr, ym, yp, zm, zp, q, cr);
    const Vec<T> aq = apply7v<T, NCP>(Q + off, j, xl, xr, ym, yp, zm, zp, q, cq);
    Vec<T> qn, f;
#pragma unroll
    for (int i = 0; i < VW; ++i) {
      qn.v[i] = cr.v[i] + bb * cq.v[i];
      f.v[i] = ar.v[i] + bb * aq.v[i];
      vt += qn.v[i] * f.v[i];
    }
    stv(Qn + off + j, qn);
    stv(F + off + j, f);
    PC_GROUPS_END
  }
  double v[1] = {(double)vt};
  block_partials<1>(v, k, blockIdx.y);
}

// F = A Q ; partial <Q|F>
template <typename T, int NCP>
__global__ void __launch_bounds__(kThreads) k_pc_apply(Blk k, PcCoef q, const T* __restrict__ Q, T* __restrict__ F) {
  if (SC(k, S_PCACT, blockIdx.y) == 0.0) return;
  T vt = T(0);
  {
    PC_GROUPS_BEGIN(k, q, T)
    Vec<T> cq;
    const Vec<T> f = apply7v<T, NCP>(Q + off, j, xl, xr, ym, yp, zm, zp, q, cq);
#pragma unroll
    for (int i = 0; i < VW; ++i) vt += cq.v[i] * f.v[i];
    stv(F + off + j, f);
    PC_GROUPS_END
  }
  double v[1] = {(double)vt};
  block_partials<1>(v, k, blockIdx.y);
}


// first step: PG = G + a Q (starting guess G); (if !last) Rn = Q - a F (Q = R0); partial |Rn|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_update1(Blk k, const T* __restrict__ G, const T* __restrict__ Q,
                                                         const T* __restrict__ F, T* __restrict__ Rn,
                                                         T* __restrict__ PG, int last) {
  GROUP_LOOP(k, T);
  if (SC(k, S_PCACT, b) == 0.0) {
    for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) stv(PG + off + gi * VW, ldv(G + off + gi * VW));
    return;
  }
  const T a = (T)SC(k, S_PCA, b);
  T vt = T(0);
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> qv = ldv(Q + e), gv = ldv(G + e);
    Vec<T> pg;
#pragma unroll
    for (int i = 0; i < VW; ++i) pg.v[i] = gv.v[i] + a * qv.v[i];
    stv(PG + e, pg);
    if (!last) {
      const Vec<T> fv = ldv(F + e);
      Vec<T> r;
#pragma unroll
      for (int i = 0; i < VW; ++i) {
        r.v[i] = qv.v[i] - a * fv.v[i];
        vt += r.v[i] * r.v[i];
      }
      stv(Rn + e, r);
    }
  }
  double v[1] = {(double)vt};
  if (!last) block_partials<1>(v, k, b);
}

// PG += a Q ; (if !last) R -= a F ; partial |R|^2
template <typename T>
__global__ void __launch_bounds__(kThreads) k_pc_update(Blk k, const T* __restrict__ Q, const T* __restrict__ F,
                                                        T* __restrict__ R, T* __restrict__ PG, int last) {
  GROUP_LOOP(k, T);
  if (SC(k, S_PCACT, b) == 0.0) return;
  const T a = (T)SC(k, S_PCA, b);
  T vt = T(0);
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> qv = ldv(Q + e);
    Vec<T> pg = ldv(PG + e);
#pragma unroll
    for (int i = 0; i < VW; ++i) pg.v[i] = pg.v[i] + a * qv.v[i];
    stv(PG + e, pg);
    if (!last) {
      const Vec<T> fv = ldv(F + e);
      Vec<T> r = ldv(R + e);
#pragma unroll
      for (int i = 0; i < VW; ++i) {
        r.v[i] = r.v[i] - a * fv.v[i];
        vt += r.v[i] * r.v[i];
      }
      stv(R + e, r);
    }
  }
  double v[1] = {(double)vt};
  if (!last) block_partials<1>(v, k, b);
}

__global__ void k_pc_sc_first(Blk k, int nu = 0) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  if (SC(k, S_ACT, b) == 0.0) {
    SC(k, S_PCACT, b) = 0.0;
    return;
  }
  const double rr1 = sum_part(k, b, 0);
  SC(k, S_RR1, b) = rr1;
  SC(k, S_PCACT, b) = rr1 < 1.0e-24 ? 0.0 : 1.0;  // cgpc_hprsdft_module.f90:181
  if (nu) {
    SC(k, S_NU0, b) = sum_part(k, b, 1);
    SC(k, S_NU1, b) = sum_part(k, b, 2);
  }
}
__global__ void k_pc_sc_alpha(Blk k) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_PCACT, b) == 0.0) return;
  const double pAp = sum_part(k, b, 0);
  SC(k, S_RR0, b) = SC(k, S_RR1, b);
  SC(k, S_PCA, b) = SC(k, S_RR0, b) / pAp;
}
__global__ void k_pc_sc_beta(Blk k) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_PCACT, b) == 0.0) return;
  const double rr1 = sum_part(k, b, 0);
  SC(k, S_RR1, b) = rr1;
  SC(k, S_PCB, b) = rr1 / SC(k, S_RR0, b);
}

// ---- s-step form of the same mloop CG steps (FP32 bands) ----
// Every vector of the preconditioner's CG lies in the Krylov space of r0 = G - A G, so it is
// evaluated in the basis v_i = B^i r0 (i < mloop), B = (A - c0 I) / c0 the off-diagonal part
// of the 7-point operator scaled to spectrum [-1, 1] (A = c0 (B + I)), with every inner
// product taken from the moments mu_j = <r0 | B^j r0>, j < 2 mloop.  The recurrence
// (alpha, beta, the update of PG) then runs on coefficient vectors per band in FP64 and the
// bands are touched in 3 mloop + 3 passes (12 for mloop = 3) instead of 26.

// Vn = B V and partials <V|Vn>, <Vn|Vn>; WRITE = false: only <V|B V>.  qb holds B's
// coefficients (c0 = 0).
template <typename T, int NCP, bool WRITE>
__global__ void __launch_bounds__(kThreads) k_pcs_shift(Blk k, PcCoef qb, const T* __restrict__ V, T* __restrict__ Vn) {
  if (SC(k, S_PCACT, blockIdx.y) == 0.0) return;
  T s0 = T(0), s1 = T(0);
  {
    PC_GROUPS_BEGIN(k, qb, T)
    Vec<T> cv;
    const Vec<T> w = apply7v<T, NCP>(V + off, j, xl, xr, ym, yp, zm, zp, qb, cv);  // qb.c0 = 0
    if (WRITE) stv(Vn + off + j, w);
#pragma unroll
    for (int i = 0; i < VW; ++i) {
      s0 += cv.v[i] * w.v[i];
      s1 += w.v[i] * w.v[i];
    }
    PC_GROUPS_END
  }
  double v[2] = {(double)s0, (double)s1};
  block_partials<2>(v, k, blockIdx.y);
}

// after the shift pass that made v_i (i >= 1): mu_{2i-1}, mu_{2i}; after the read-only pass
// (i = m): mu_{2m-1}, then the CG recurrence on coefficients, leaving xi_0 .. xi_{m-1}
__global__ void k_pcs_sc(Blk k, int i, int m, double c0) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_PCACT, b) == 0.0) return;
  if (i == 0) {  // after k_pc_first
    SC(k, S_MU0, b) = SC(k, S_RR1, b);
    return;
  }
  SC(k, S_MU0 + 2 * i - 1, b) = sum_part(k, b, 0);
  if (i < m) {
    SC(k, S_MU0 + 2 * i, b) = sum_part(k, b, 1);
    return;
  }
  double mu[8], xi[5];
  for (int j = 0; j < 2 * m; ++j) mu[j] = SC(k, S_MU0 + j, b);
  pcs_recurrence(mu, m, c0, xi);
  for (int j = 0; j < m; ++j) SC(k, S_XI0 + j, b) = xi[j];
}

// PG = G + sum_{i < M} xi_i v_i (PG = G where the preconditioner is inactive), and the
// partial <PG|G> that CG takes next (bands CG still updates)
template <typename T, int M>
__global__ void __launch_bounds__(kThreads) k_pcs_combine(Blk k, const T* __restrict__ G, const T* __restrict__ V0,
                                                          const T* __restrict__ V1, const T* __restrict__ V2,
                                                          const T* __restrict__ V3, T* __restrict__ PG) {
  GROUP_LOOP(k, T);
  const bool on = SC(k, S_PCACT, b) != 0.0;
  T x[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) x[j] = (on && j < M) ? (T)SC(k, S_XI0 + j, b) : T(0);
  double vt = 0.0;  // accumulated as k_dot does
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    const Vec<T> gv = ldv(G + e);
    Vec<T> pv = gv;
    if (on) {
      const Vec<T> a0 = ldv(V0 + e);
#pragma unroll
      for (int i = 0; i < VW; ++i) pv.v[i] += x[0] * a0.v[i];
      if (M > 1) {
        const Vec<T> a1 = ldv(V1 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[1] * a1.v[i];
      }
      if (M > 2) {
        const Vec<T> a2 = ldv(V2 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[2] * a2.v[i];
      }
      if (M > 3) {
        const Vec<T> a3 = ldv(V3 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[3] * a3.v[i];
      }
    }
    stv(PG + e, pv);
#pragma unroll
    for (int i = 0; i < VW; ++i) vt += (double)pv.v[i] * (double)gv.v[i];
  }
  if (SC(k, S_ACT, b) == 0.0) return;
  double d[1] = {vt};
  block_partials<1>(d, k, b);
}

// CG's rb = <PG|G> dV and beta = rb / gkgk (k_sc_beta) without a pass over PG:
// <PG|G> = <G|G> + sum_i xi_i nu_i with nu_i = <B^i v0|G>.  nu_0 and nu_1 come from k_pc_first;
// since v0 = G - A G = (1 - c0) G - c0 B G, nu_{i+1} = ((1 - c0) nu_i - mu_i) / c0 for the
// rest.  <G|G> dV is the rb CG left in S_RB (k_sc_rb, k_sc_reject).
__global__ void k_pcs_beta(Blk k, int m, double c0, double dV, int first) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb || SC(k, S_ACT, b) == 0.0) return;
  double pgg = SC(k, S_RB, b) / dV;
  if (SC(k, S_PCACT, b) != 0.0) {
    double nu[4];
    nu[0] = SC(k, S_NU0, b);
    nu[1] = SC(k, S_NU1, b);
    for (int i = 2; i < m; ++i) nu[i] = ((1.0 - c0) * nu[i - 1] - SC(k, S_MU0 + i - 1, b)) / c0;
    for (int i = 0; i < m; ++i) pgg += SC(k, S_XI0 + i, b) * nu[i];
  }
  const double rb = pgg * dV;
  SC(k, S_RB, b) = rb;
  SC(k, S_BETA, b) = first ? 0.0 : rb / SC(k, S_GKGK, b);
  SC(k, S_GKGK, b) = rb;
}

// P = PG + beta P with PG = G + sum_{i < M} xi_i v_i (P = PG at the first CG step; PG = G where
// the preconditioner is inactive), i.e. k_pcs_combine and k_make_p in one pass; bands whose CG
// has stopped keep P
template <typename T, int M>
__global__ void __launch_bounds__(kThreads) k_pcs_combine_p(Blk k, const T* __restrict__ G, const T* __restrict__ V0,
                                                            const T* __restrict__ V1, const T* __restrict__ V2,
                                                            const T* __restrict__ V3, T* __restrict__ P, int first) {
  GROUP_LOOP(k, T);
  if (SC(k, S_ACT, b) == 0.0) return;
  const bool on = SC(k, S_PCACT, b) != 0.0;
  T x[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) x[j] = (on && j < M) ? (T)SC(k, S_XI0 + j, b) : T(0);
  const T beta = (T)SC(k, S_BETA, b);
  for (size_t gi = g0 + threadIdx.x; gi < g1; gi += kThreads) {
    const size_t e = off + gi * VW;
    Vec<T> pv = ldv(G + e);
    if (on) {
      const Vec<T> a0 = ldv(V0 + e);
#pragma unroll
      for (int i = 0; i < VW; ++i) pv.v[i] += x[0] * a0.v[i];
      if (M > 1) {
        const Vec<T> a1 = ldv(V1 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[1] * a1.v[i];
      }
      if (M > 2) {
        const Vec<T> a2 = ldv(V2 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[2] * a2.v[i];
      }
      if (M > 3) {
        const Vec<T> a3 = ldv(V3 + e);
#pragma unroll
        for (int i = 0; i < VW; ++i) pv.v[i] += x[3] * a3.v[i];
      }
    }
    if (!first) {
      const Vec<T> po = ldv(P + e);
#pragma unroll
      for (int i = 0; i < VW; ++i) pv.v[i] += beta * po.v[i];
    }
    stv(P + e, pv);
  }
}

// ---------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------
// CTAs (chunks) per band of the elementwise and preconditioner passes.  Large planes (more than
// 4096 reals, e.g. 128^2): one z plane per chunk, so that the z neighbours of a chunk's rows are
// rows that neighbouring CTAs stream at the same time (L2 hits); measured at c3 the
// preconditioner passes take 23 % less time than with 4-plane chunks.  Smaller grids: chunks of
// about 4096 reals, at most 16 x 148 x 4 CTAs in all (measured best at c1, 64^2 planes).
static int pick_nch(size_t ng, int nbb, int plane_reals = 0, int n3 = 0) {
  if (plane_reals > 4096 && n3 >= 1 && n3 <= kMaxChunks && (long long)n3 * nbb <= 64LL * 148 * 4) return n3;
  int nch = (int)std::min<size_t>(kMaxChunks, (ng + 4095) / 4096);
  while (nch > 1 && (long long)nch * nbb > 16 * 148 * 4) nch /= 2;
  return std::max(1, nch);
}

#define LAUNCH_E(kern, ...)                                                  \
  do {                                                                       \
    kern<<<dim3(k.nch, k.nbb), kThreads, 0, c.stream>>>(k, __VA_ARGS__);     \
    c.launches++;                                                            \
  } while (0)
#define LAUNCH_S(kern, ...)                                                  \
  do {                                                                       \
    kern<<<(k.nbb + 127) / 128, 128, 0, c.stream>>>(k, ##__VA_ARGS__);       \
    c.launches++;                                                            \
  } while (0)

// precond_hprsdft (cgpc_hprsdft_module.f90:133-270) on a band block: PG = G + sum_it a_it Q_it
// for mloop CG steps on A x = G from x = G.  Buffers: X0 holds R0 = Q1, then X0/X1/X2 rotate
// between the residual and the current/next directions; F = A Q.
// *pg_dot: set when the partials of <PG|G> (bands with S_ACT set) were left in the partial
// buffer by the last pass.  P (s-step form only; p_done is set when it was used): the CG
// direction P = PG + beta P (first: P = PG) is formed by the last pass instead of PG, with rb
// and beta set as k_sc_beta sets them.
template <typename T>
static int pc_block(Ctx& c, Blk& k, const T* G, T* PG, T* X0, T* X1, T* X2, T* F, bool* pg_dot = nullptr,
                    T* P = nullptr, int first = 0, bool* p_done = nullptr) {
  if (pg_dot) *pg_dot = false;
  if (p_done) *p_done = false;
  PcCoef q;
  const double* H = c.p.hgrid;
  q.c0 = c.p.ggg[0] / (H[0] * H[0]) + c.p.ggg[1] / (H[1] * H[1]) + c.p.ggg[2] / (H[2] * H[2]);
  q.c1 = -0.5 * c.p.ggg[0] / (H[0] * H[0]);
  q.c2 = -0.5 * c.p.ggg[1] / (H[1] * H[1]);
  q.c3 = -0.5 * c.p.ggg[2] / (H[2] * H[2]);
  q.n1 = c.p.n1; q.n2 = c.p.n2; q.n3 = c.p.n3;
  q.nc = c.cplx ? 2 : 1;
  RS_CHECK((q.n1 * q.nc) % Vec<T>::W == 0, RSDFT_ERR_UNSUPPORTED,
           "preconditioner needs x-rows of a multiple of %d reals", Vec<T>::W);
  ProfScope ps(c, "pc");
  // kernels on rows of n1 * nc reals: real (1) or complex (2) interleaved view
#define LAUNCH_PC(kern, ...)                                   \
  do {                                                         \
    if (q.nc == 1) LAUNCH_E((kern<T, 1>), __VA_ARGS__);        \
    else LAUNCH_E((kern<T, 2>), __VA_ARGS__);                  \
  } while (0)
  if (c.p.mloop < 1) {
    LAUNCH_E(k_copy<T>, G, PG);
    return check_launch("pc");
  }
  if (std::is_same<T, float>::value && c.pc_sstep && c.p.mloop <= 4) {
    // s-step form (FP32 bands): v0 = R0 in X0, v1 = B v0 in X1, v2 in X2, v3 in F
    const int m = c.p.mloop;
    PcCoef qb = q;
    qb.c1 = q.c1 / q.c0;
    qb.c2 = q.c2 / q.c0;
    qb.c3 = q.c3 / q.c0;
    qb.c0 = 0.0;
    T* v[4] = {X0, X1, X2, F};
    const bool direct = P != nullptr && p_done != nullptr;
    if (direct) {
      if (q.nc == 1) LAUNCH_E((k_pc_first<T, 1, true>), q, G, X0);
      else LAUNCH_E((k_pc_first<T, 2, true>), q, G, X0);
    } else {
      LAUNCH_PC(k_pc_first, q, G, X0);
    }
    LAUNCH_S(k_pc_sc_first, direct ? 1 : 0);
    LAUNCH_S(k_pcs_sc, 0, m, q.c0);
    for (int i = 1; i < m; ++i) {
      if (q.nc == 1) LAUNCH_E((k_pcs_shift<T, 1, true>), qb, v[i - 1], v[i]);
      else LAUNCH_E((k_pcs_shift<T, 2, true>), qb, v[i - 1], v[i]);
      LAUNCH_S(k_pcs_sc, i, m, q.c0);
    }
    if (q.nc == 1) LAUNCH_E((k_pcs_shift<T, 1, false>), qb, v[m - 1], (T*)nullptr);
    else LAUNCH_E((k_pcs_shift<T, 2, false>), qb, v[m - 1], (T*)nullptr);
    LAUNCH_S(k_pcs_sc, m, m, q.c0);
    if (direct) {
      LAUNCH_S(k_pcs_beta, m, q.c0, c.p.dv, first);
      switch (m) {
        case 1: LAUNCH_E((k_pcs_combine_p<T, 1>), G, v[0], v[1], v[2], v[3], P, first); break;
        case 2: LAUNCH_E((k_pcs_combine_p<T, 2>), G, v[0], v[1], v[2], v[3], P, first); break;
        case 3: LAUNCH_E((k_pcs_combine_p<T, 3>), G, v[0], v[1], v[2], v[3], P, first); break;
        default: LAUNCH_E((k_pcs_combine_p<T, 4>), G, v[0], v[1], v[2], v[3], P, first); break;
      }
      *p_done = true;
      return check_launch("pc");
    }
    switch (m) {
      case 1: LAUNCH_E((k_pcs_combine<T, 1>), G, v[0], v[1], v[2], v[3], PG); break;
      case 2: LAUNCH_E((k_pcs_combine<T, 2>), G, v[0], v[1], v[2], v[3], PG); break;
      case 3: LAUNCH_E((k_pcs_combine<T, 3>), G, v[0], v[1], v[2], v[3], PG); break;
      default: LAUNCH_E((k_pcs_combine<T, 4>), G, v[0], v[1], v[2], v[3], PG); break;
    }
    if (pg_dot) *pg_dot = true;
    return check_launch("pc");
  }
  LAUNCH_PC(k_pc_first, q, G, X0);
  LAUNCH_S(k_pc_sc_first);
  LAUNCH_PC(k_pc_apply, q, X0, F);
  LAUNCH_S(k_pc_sc_alpha);
  LAUNCH_E(k_pc_update1<T>, G, X0, F, X1, PG, c.p.mloop == 1 ? 1 : 0);
  T* r = X1;   // residual
  T* qo = X0;  // current direction
  T* qn = X2;  // next direction
  for (int it = 2; it <= c.p.mloop; ++it) {
    LAUNCH_S(k_pc_sc_beta);
    LAUNCH_PC(k_pc_dirapply, q, r, qo, qn, F);
    LAUNCH_S(k_pc_sc_alpha);
    const int last = it == c.p.mloop;
    LAUNCH_E(k_pc_update<T>, qn, F, r, PG, last);
    std::swap(qo, qn);
  }
#undef LAUNCH_PC
  return check_launch("pc");
}

template <typename T>
int precond_real(Ctx& c, const T* g, T* pg, size_t ld, int nb) {
  const size_t nreal = c.ng * (c.cplx ? 2 : 1);
  RS_CHECK(ld == nreal, RSDFT_ERR_ARG, "precond: ld must equal the grid size");
  Blk k;
  k.nbb = nb;
  k.ng = nreal;
  k.nch = pick_nch(nreal, nb, c.p.n1 * c.p.n2 * (c.cplx ? 2 : 1), c.p.n3);
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nb + 64));
  RS_TRY(c.ws_red.ensure(sizeof(double) * kPS * (size_t)nb * k.nch));
  RS_TRY(c.ws_cg.ensure(sizeof(T) * 4 * nreal * (size_t)nb));
  k.sc = c.ws_scal.as<double>();
  k.part = c.ws_red.as<double>();
  std::vector<double> act((size_t)nb, 1.0);
  RS_CUDA(cudaMemcpyAsync(k.sc + (size_t)S_ACT * nb, act.data(), sizeof(double) * nb, cudaMemcpyHostToDevice,
                          c.stream));
  T* X0 = c.ws_cg.as<T>();
  T* X1 = X0 + nreal * nb;
  T* X2 = X1 + nreal * nb;
  T* F = X2 + nreal * nb;
  RS_TRY(pc_block<T>(c, k, g, pg, X0, X1, X2, F));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}
template int precond_real<double>(Ctx&, const double*, double*, size_t, int);
template int precond_real<float>(Ctx&, const float*, float*, size_t, int);

// ---------------------------------------------------------------------------
// cggs (src/conjugate_gradient/cggs_module.f90:14-124, called after the preconditioner at
// src/conjugate_gradient/cg_module.f90:249-251 and :576-578): the preconditioned gradient of band
// n loses its components along the current bands m (m < n: iswitch 1, cggs_1; m != n:
// iswitch 2, cggs_2), classical Gram-Schmidt: all projections dV <x_m|Pg_n> first, then
// Pg_n -= sum_m x_m <x_m|Pg_n> dV.  Bands of earlier CG blocks hold their final values, bands of
// the current block their values at this CG step (the reference's MB_d block semantics).
// The two products are plain library GEMMs (cuBLAS, in the storage precision).
// ---------------------------------------------------------------------------
// C (range x nn, column-major, NC reals per element): keep entry (m, j) where band m may be
// projected out of band b0 + j, negated; zero elsewhere
template <typename T, int NC>
__global__ void k_cggs_mask(T* C, int range, int nn, int b0, int iswitch) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)range * nn;
       t += (long long)gridDim.x * blockDim.x) {
    const int m = (int)(t % range), j = (int)(t / range), n = b0 + j;
    const bool keep = iswitch == 1 ? m < n : m != n;
#pragma unroll
    for (int q = 0; q < NC; ++q) C[t * NC + q] = keep ? -C[t * NC + q] : T(0);
  }
}

#define RS_CUBLAS_CG(call)                                                        \
  do {                                                                            \
    cublasStatus_t st_ = (call);                                                  \
    RS_CHECK(st_ == CUBLAS_STATUS_SUCCESS, RSDFT_ERR_CUDA, "%s -> cuBLAS status %d", #call, (int)st_); \
  } while (0)

template <typename T, int NC>
static int cggs_block(Ctx& c, const T* psi, int nb, int b0, int nn, T* PG) {
  const int range = c.cggs == 1 ? b0 + nn : nb;
  if (range <= 0 || nn <= 0) return 0;
  const int ng = (int)c.ng;
  RS_TRY(c.ws_dense.ensure(sizeof(T) * NC * (size_t)range * nn));
  T* C = c.ws_dense.as<T>();
  ProfScope ps(c, "cg");
  if (NC == 1 && std::is_same<T, double>::value) {
    const double dV = c.p.dv, zero = 0.0, one = 1.0;
    const double* X = reinterpret_cast<const double*>(psi);
    double* Pd = reinterpret_cast<double*>(PG);
    double* Cd = reinterpret_cast<double*>(C);
    RS_CUBLAS_CG(cublasDgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, range, nn, ng, &dV, X, ng, Pd, ng, &zero, Cd, range));
    k_cggs_mask<double, 1><<<64, 256, 0, c.stream>>>(Cd, range, nn, b0, c.cggs);
    c.launches++;
    RS_CUBLAS_CG(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, ng, nn, range, &one, X, ng, Cd, range, &one, Pd, ng));
  } else if (NC == 1) {
    const float dV = (float)c.p.dv, zero = 0.f, one = 1.f;
    const float* X = reinterpret_cast<const float*>(psi);
    float* Pf = reinterpret_cast<float*>(PG);
    float* Cf = reinterpret_cast<float*>(C);
    RS_CUBLAS_CG(cublasSgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, range, nn, ng, &dV, X, ng, Pf, ng, &zero, Cf, range));
    k_cggs_mask<float, 1><<<64, 256, 0, c.stream>>>(Cf, range, nn, b0, c.cggs);
    c.launches++;
    RS_CUBLAS_CG(cublasSgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, ng, nn, range, &one, X, ng, Cf, range, &one, Pf, ng));
  } else if (std::is_same<T, double>::value) {
    const cuDoubleComplex dV = make_cuDoubleComplex(c.p.dv, 0.0), zero = make_cuDoubleComplex(0.0, 0.0),
                          one = make_cuDoubleComplex(1.0, 0.0);
    const cuDoubleComplex* X = reinterpret_cast<const cuDoubleComplex*>(psi);
    cuDoubleComplex* Pz = reinterpret_cast<cuDoubleComplex*>(PG);
    cuDoubleComplex* Cz = reinterpret_cast<cuDoubleComplex*>(C);
    RS_CUBLAS_CG(cublasZgemm(c.cublas, CUBLAS_OP_C, CUBLAS_OP_N, range, nn, ng, &dV, X, ng, Pz, ng, &zero, Cz, range));
    k_cggs_mask<double, 2><<<64, 256, 0, c.stream>>>(reinterpret_cast<double*>(C), range, nn, b0, c.cggs);
    c.launches++;
    RS_CUBLAS_CG(cublasZgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, ng, nn, range, &one, X, ng, Cz, range, &one, Pz, ng));
  } else {
    const cuComplex dV = make_cuComplex((float)c.p.dv, 0.f), zero = make_cuComplex(0.f, 0.f), one = make_cuComplex(1.f, 0.f);
    const cuComplex* X = reinterpret_cast<const cuComplex*>(psi);
    cuComplex* Pc = reinterpret_cast<cuComplex*>(PG);
    cuComplex* Cc = reinterpret_cast<cuComplex*>(C);
    RS_CUBLAS_CG(cublasCgemm(c.cublas, CUBLAS_OP_C, CUBLAS_OP_N, range, nn, ng, &dV, X, ng, Pc, ng, &zero, Cc, range));
    k_cggs_mask<float, 2><<<64, 256, 0, c.stream>>>(reinterpret_cast<float*>(C), range, nn, b0, c.cggs);
    c.launches++;
    RS_CUBLAS_CG(cublasCgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, ng, nn, range, &one, X, ng, Cc, range, &one, Pc, ng));
  }
  return check_launch("cggs");
}

template <typename T>
static int hpsi_any(Ctx& c, int kk, int s, const T* x, T* hx, size_t ld, int nb) {
  if (c.cplx) return hpsi_cplx<T>(c, kk, s, x, hx, ld, nb);
  return hpsi_real<T>(c, kk, s, x, hx, ld, nb);
}

// Preconditioner CG uses now: the learned one only where it is built (real build, FP32
// bands) and trained; otherwise precond_hprsdft stands in.
int pc_effective(const Ctx& c) {
  if (c.pc_cur == RSDFT_PC_LEARNED && !(lpc_ready() && c.mixed && !c.cplx)) return RSDFT_PC_HPRSDFT;
  return c.pc_cur;
}

template <typename T, int NC>
static int cg_block_run(Ctx& c, int kk, int s, double* h_esp, double* h_res) {
  const int nb = c.kp[kk].nband;
  const size_t nreal = c.ng * NC;
  RS_CHECK(nreal % Vec<T>::W == 0, RSDFT_ERR_UNSUPPORTED, "CG needs bands of a multiple of %d reals", Vec<T>::W);
  int nbb = c.p.cg_block > 0 ? std::min(c.p.cg_block, nb) : nb;
  // real build: H x of all bands lives in ws_hpsi, where the fused GS/SD step that follows in
  // the sweep finds it; the other eight vectors per band are block workspace
  c.cg_hx_ready = false;
  T* HXall = nullptr;
  if (NC == 1) {
    RS_TRY(c.ws_hpsi.ensure(sizeof(T) * nreal * (size_t)nb));
    HXall = c.ws_hpsi.as<T>();
  }
  RS_TRY(c.ws_flag.ensure(sizeof(int) * 4));
  RS_CUDA(cudaMemsetAsync(c.ws_flag.p, 0, sizeof(int), c.stream));
  size_t freeb = 0, totb = 0;
  cudaMemGetInfo(&freeb, &totb);
  const size_t per_band = (HXall ? 8 : 9) * nreal * sizeof(T);
  const size_t budget = (size_t)(0.4 * (double)(freeb + c.ws_cg.bytes));
  if (c.p.cg_block <= 0)
    while (nbb > 1 && (size_t)nbb * per_band > budget) nbb = (nbb + 1) / 2;
  RS_TRY(c.ws_cg.ensure(per_band * nbb));
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nbb + 64));
  Blk k;
  k.ng = nreal;
  k.nch = pick_nch(nreal, nbb, c.p.n1 * c.p.n2 * NC, c.p.n3);
  RS_TRY(c.ws_red.ensure(sizeof(double) *
                         std::max<size_t>(kPS * (size_t)nbb * pick_nch(nreal, 1), pc_fused_part_doubles(c, nbb))));
  k.sc = c.ws_scal.as<double>();
  k.part = c.ws_red.as<double>();
  T* base = c.ws_cg.as<T>();
  T* HX = HXall ? nullptr : base;
  T* HP = HXall ? base : HX + nreal * nbb;
  T* G = HP + nreal * nbb;
  T* PG = G + nreal * nbb;
  T* P = PG + nreal * nbb;
  T* R = P + nreal * nbb;
  T* Q = R + nreal * nbb;
  T* Q2 = Q + nreal * nbb;
  T* F = Q2 + nreal * nbb;
  T* psi = c.wfn(kk, s).psi.as<T>();
  const double dV = c.p.dv;
  // real build: g = -2(Hx - Ex), res = rb/2^2; complex build: g = -(Hx - Ex), res = rb
  const double gfac = NC == 1 ? -2.0 : -1.0, c1sq = NC == 1 ? 4.0 : 1.0;
  std::vector<double> hE, hR;
  for (int b0 = 0; b0 < nb; b0 += nbb) {
    const int nn = std::min(nbb, nb - b0);
    k.nbb = nn;
    k.nch = pick_nch(nreal, nn, c.p.n1 * c.p.n2 * NC, c.p.n3);
    T* X = psi + (size_t)b0 * nreal;
    if (HXall) HX = HXall + (size_t)b0 * nreal;
    RS_TRY(hpsi_any<T>(c, kk, s, X, HX, nreal, nn));
    {
      ProfScope ps(c, "cg");
      LAUNCH_E(k_dot<T>, X, HX, -1);
      LAUNCH_S(k_sc_init, dV);
      LAUNCH_E(k_make_g<T>, X, HX, G, gfac);
      LAUNCH_S(k_sc_rb, dV);
    }
    for (int icg = 1; icg <= c.p.ncg + 1; ++icg) {
      {
        ProfScope ps(c, "cg");
        LAUNCH_S(k_sc_top, c1sq);
      }
      if (icg == c.p.ncg + 1) break;
      const int pcm = pc_effective(c);
      bool pg_dot = false;  // <PG|G> partials already formed by the preconditioner's last pass
      bool p_done = false;  // rb, beta and p already formed by the fused preconditioner
      if (pcm == RSDFT_PC_HPRSDFT && std::is_same<T, float>::value && pc_fused_applies(c)) {
        RS_TRY(pc_fused_step(c, k, reinterpret_cast<const float*>(G), reinterpret_cast<float*>(P), icg == 1 ? 1 : 0));
        p_done = true;
      } else if (pcm == RSDFT_PC_NONE) {
        ProfScope ps(c, "cg");
        LAUNCH_E(k_copy<T>, G, PG);
      } else if (pcm == RSDFT_PC_LEARNED && std::is_same<T, float>::value && NC == 1) {
        RS_TRY(lpc_apply(c, reinterpret_cast<const float*>(G), reinterpret_cast<float*>(PG), nn));
      } else if (c.pc_direct && !c.cggs) {
        // the s-step form writes P itself (its direction pass replaces k_make_p)
        RS_TRY(pc_block<T>(c, k, G, PG, R, Q, Q2, F, &pg_dot, P, icg == 1 ? 1 : 0, &p_done));
      } else {
        RS_TRY(pc_block<T>(c, k, G, PG, R, Q, Q2, F, &pg_dot));
      }
      if (c.cggs) {
        // inactive bands' gradients are left alone: their CG has stopped (the reference leaves
        // its icg loop before the preconditioner for them)
        RS_TRY((cggs_block<T, NC>(c, psi, nb, b0, nn, PG)));
        pg_dot = false;
      }
      if (!p_done) {
        ProfScope ps(c, "cg");
        if (!pg_dot) LAUNCH_E(k_dot<T>, PG, G, (int)S_ACT);
        LAUNCH_S(k_sc_beta, dV, icg == 1 ? 1 : 0);
        LAUNCH_E(k_make_p<T>, PG, P, icg == 1 ? 1 : 0);
      }
      RS_TRY(hpsi_any<T>(c, kk, s, P, HP, nreal, nn));
      {
        ProfScope ps(c, "cg");
        LAUNCH_E((k_dots6<T, NC>), X, P, HX, HP);
        LAUNCH_S(k_sc_solve2<NC>, dV);
        LAUNCH_E((k_update_hg<T, NC>), X, P, HX, HP, G, gfac);
        LAUNCH_S(k_sc_reject, dV, c.ws_flag.as<int>());
        LAUNCH_E((k_update_x<T, NC>), X, P);
      }
    }
    RS_TRY(check_launch("cg"));
    if (h_esp || h_res) {
      hE.resize(nn);
      hR.resize(nn);
      RS_CUDA(cudaMemcpyAsync(hE.data(), k.sc + (size_t)S_E * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost,
                              c.stream));
      RS_CUDA(cudaMemcpyAsync(hR.data(), k.sc + (size_t)S_RES * nn, sizeof(double) * nn, cudaMemcpyDeviceToHost,
                              c.stream));
      RS_CUDA(cudaStreamSynchronize(c.stream));
      if (h_esp) std::memcpy(h_esp + b0, hE.data(), sizeof(double) * nn);
      if (h_res) std::memcpy(h_res + b0, hR.data(), sizeof(double) * nn);
    }
  }
  if (HXall) {
    c.cg_hx_ready = true;
    c.cg_hx_k = kk;
    c.cg_hx_s = s;
  }
  return 0;
}

int cg_run(Ctx& c, int k, int s, double* h_esp, double* h_res) {
  if (c.cplx) return c.mixed ? cg_block_run<float, 2>(c, k, s, h_esp, h_res) : cg_block_run<double, 2>(c, k, s, h_esp, h_res);
  return c.mixed ? cg_block_run<float, 1>(c, k, s, h_esp, h_res) : cg_block_run<double, 1>(c, k, s, h_esp, h_res);
}

// ---------------------------------------------------------------------------
// FP64 residual check (esp_calc + the CG residual definition, in FP64 for any storage)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) k_res_dots(Blk k, const T* __restrict__ x, const double* __restrict__ hx) {
  BAND_LOOP(k, 1);
  double v[2] = {0.0, 0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double xi = (double)x[off + i];
    v[0] += xi * xi;
    v[1] += xi * hx[off + i];
  }
  block_partials<2>(v, k, b);
}
__global__ void k_res_sc1(Blk k, double* esp) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  const double xx = sum_part(k, b, 0), xh = sum_part(k, b, 1);
  SC(k, S_RR0, b) = xx;
  SC(k, S_E, b) = xh / xx;
  esp[b] = xh / xx;
}
template <typename T>
__global__ void __launch_bounds__(kThreads) k_res_norm(Blk k, const T* __restrict__ x, const double* __restrict__ hx) {
  BAND_LOOP(k, 1);
  const double e = SC(k, S_E, b);
  double v[1] = {0.0};
  for (size_t i = i0 + threadIdx.x; i < i1; i += kThreads) {
    const double r = hx[off + i] - e * (double)x[off + i];
    v[0] += r * r;
  }
  block_partials<1>(v, k, b);
}
__global__ void k_res_sc2(Blk k, double* res) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= k.nbb) return;
  res[b] = sum_part(k, b, 0) / SC(k, S_RR0, b);
}

template <typename T>
static int residual_t(Ctx& c, int kk, int s, double* d_esp, double* d_res) {
  const int nb = c.kp[kk].nband;
  const int nc = c.cplx ? 2 : 1;
  const size_t nreal = c.ng * nc;
  // band chunk so that the FP64 copies stay around 1 GiB
  int nbc = (int)std::max<size_t>(1, std::min<size_t>(nb, (size_t)(1u << 30) / (16 * nreal)));
  const size_t extra = std::is_same<T, double>::value ? 0 : 1;
  RS_TRY(c.ws_rot.ensure(sizeof(double) * nreal * nbc * (1 + extra)));
  RS_TRY(c.ws_scal.ensure(sizeof(double) * S_COUNT * nbc + 64));
  const T* psi = c.wfn(kk, s).psi.as<T>();
  double* HX = c.ws_rot.as<double>();
  double* XD = HX + nreal * nbc;
  Blk k;
  k.ng = nreal;
  for (int b0 = 0; b0 < nb; b0 += nbc) {
    const int nn = std::min(nbc, nb - b0);
    k.nbb = nn;
    k.nch = pick_nch(nreal, nn);
    RS_TRY(c.ws_red.ensure(sizeof(double) * kPS * (size_t)nn * k.nch));
    k.sc = c.ws_scal.as<double>();
    k.part = c.ws_red.as<double>();
    const T* X = psi + (size_t)b0 * nreal;
    const double* XH;
    if (std::is_same<T, double>::value) {
      XH = reinterpret_cast<const double*>(X);
    } else {
      RS_TRY(convert_f2d(c, reinterpret_cast<const float*>(X), XD, nreal * nn));
      XH = XD;
    }
    RS_TRY(hpsi_any<double>(c, kk, s, XH, HX, nreal, nn));
    ProfScope ps(c, "residual");
    LAUNCH_E(k_res_dots<T>, X, HX);
    LAUNCH_S(k_res_sc1, d_esp + b0);
    LAUNCH_E(k_res_norm<T>, X, HX);
    LAUNCH_S(k_res_sc2, d_res + b0);
  }
  return check_launch("residual");
}

int residual_run(Ctx& c, int k, int s, double* d_esp, double* d_res) {
  if (c.mixed) return residual_t<float>(c, k, s, d_esp, d_res);
  return residual_t<double>(c, k, s, d_esp, d_res);
}

}  // namespace rsdft
