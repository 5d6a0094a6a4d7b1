// GGA-PBE exchange-correlation potential on the device, for the SCF loop of structures read
// from pseudopotential files.
//
// Reference (restated, not translated): calc_GGAPBE96_2 (src/xc/xc_ggapbe96_2_module.f90:26-370)
// with mu = 0.21951, kappa = 0.804, beta = 3 mu / pi^2; densities at or below 1e-10 are skipped;
// the gradient is that of the total density (construct_gradient16, src/kinetic/gradient_module.f90:
// 92-175, central FD of order Md), used in the exchange of each spin and in the correlation; the
// divergence terms are the FD derivative of the flux scaled by 1/H (calc_abc_gradient_org,
// :349-438); where a spin's density is below the cut, its exchange flux factor keeps the value of
// the previous spin at that point, as the reference's loop leaves it.
//
// Three passes over the grid: the gradient of the total density; the pointwise PBE terms
// (local potentials, the flux (r_x,s + r_c) grad(rho) / H per spin and axis, energy partials);
// the divergence of the fluxes.  FP64 throughout; the energy partials are summed per block and
// added in a fixed order on the host.
#include <cmath>
#include <vector>

#include "ctx.cuh"

namespace rsdft {
namespace {

constexpr int kXcThreads = 256;
constexpr int kXcBlocks = 2 * 148;
constexpr int kXcMdMax = 6;

struct XcGrid {
  int n1, n2, n3, md;
  double ih[3];                 // 1 / H per axis
  double nab[kXcMdMax + 1];     // nab(1..md)
};

__device__ __forceinline__ size_t xc_idx(int x, int y, int z, const XcGrid& g) {
  return (size_t)x + (size_t)g.n1 * ((size_t)y + (size_t)g.n2 * (size_t)z);
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

// gradient of the total density rho[0] (+ rho[1]): sum_m nab(m) (t(i + m) - t(i - m)) / H
__global__ void __launch_bounds__(kXcThreads) k_xc_grad(const double* __restrict__ rho, int ns, XcGrid g,
                                                        double* __restrict__ gx, double* __restrict__ gy,
                                                        double* __restrict__ gz) {
  const size_t ng = (size_t)g.n1 * g.n2 * g.n3;
  for (size_t i = blockIdx.x * (size_t)kXcThreads + threadIdx.x; i < ng; i += (size_t)gridDim.x * kXcThreads) {
    const int x = (int)(i % g.n1), y = (int)((i / g.n1) % g.n2), z = (int)(i / ((size_t)g.n1 * g.n2));
    double d[3] = {0.0, 0.0, 0.0};
    for (int m = 1; m <= g.md; ++m) {
      const size_t ip[3] = {xc_idx(wrap(x + m, g.n1), y, z, g), xc_idx(x, wrap(y + m, g.n2), z, g),
                            xc_idx(x, y, wrap(z + m, g.n3), g)};
      const size_t im[3] = {xc_idx(wrap(x - m, g.n1), y, z, g), xc_idx(x, wrap(y - m, g.n2), z, g),
                            xc_idx(x, y, wrap(z - m, g.n3), g)};
      for (int a = 0; a < 3; ++a) {
        double tp = rho[ip[a]], tm = rho[im[a]];
        if (ns == 2) {
          tp += rho[ng + ip[a]];
          tm += rho[ng + im[a]];
        }
        d[a] += g.nab[m] * (tp - tm);
      }
    }
    gx[i] = d[0] * g.ih[0];
    gy[i] = d[1] * g.ih[1];
    gz[i] = d[2] * g.ih[2];
  }
}

__device__ __forceinline__ void xc_block_sum2(double a, double b, double* part) {
  __shared__ double red[2][kXcThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int w = 0; w < kXcThreads / 32; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
    }
    part[2 * blockIdx.x] = s0;
    part[2 * blockIdx.x + 1] = s1;
  }
}

// PW92 correlation energy per particle of one spin channel fit and its rs derivative
__device__ __forceinline__ void pw92(double A, double alp, double b1, double b2, double b3, double b4, double rs,
                                     double rssq, double& e, double& de) {
  const double q = b1 * rssq + b2 * rs + b3 * rs * rssq + b4 * rs * rs;
  e = -2.0 * A * (1.0 + alp * rs) * log(1.0 + 1.0 / (2.0 * A * q));
  de = alp * e / (1.0 + alp * rs) +
       A * (1.0 + alp * rs) / rssq * (b1 + 2.0 * b2 * rssq + 3.0 * b3 * rs + 4.0 * b4 * rs * rssq) / (2.0 * A * q * q + q);
}

// pointwise PBE: vloc[s] local terms, flux[s][a] = (r_x,s + r_c) g_a / H_a, energy partials
__global__ void __launch_bounds__(kXcThreads) k_xc_pbe(const double* __restrict__ rho, int ns, XcGrid g, double mu,
                                                       double kp, const double* __restrict__ gx,
                                                       const double* __restrict__ gy, const double* __restrict__ gz,
                                                       double* __restrict__ vloc, double* __restrict__ flux,
                                                       double* __restrict__ part) {
  const size_t ng = (size_t)g.n1 * g.n2 * g.n3;
  const double pi = 3.14159265358979323846;
  const double beta = mu * 3.0 / (pi * pi);
  const double const1 = pow(2.0, 4.0 / 3.0) - 2.0;
  const double const2 = 9.0 * (pow(2.0, 1.0 / 3.0) - 1.0) / 4.0;
  const double C2 = (1.0 - log(2.0)) / (pi * pi);
  const double C1 = beta / C2;
  double ex_sum = 0.0, ec_sum = 0.0;
  for (size_t i = blockIdx.x * (size_t)kXcThreads + threadIdx.x; i < ng; i += (size_t)gridDim.x * kXcThreads) {
    const double gxi = gx[i], gyi = gy[i], gzi = gz[i];
    const double gg = gxi * gxi + gyi * gyi + gzi * gzi;
    // exchange, each spin with trho = 2 rho_s (one spin: rho)
    const double factor = ns == 2 ? 2.0 : 1.0;
    double rtx[2] = {0.0, 0.0}, vx[2] = {0.0, 0.0};
    double rt = 0.0;
    for (int s = 0; s < ns; ++s) {
      const double trho = factor * rho[(size_t)s * ng + i];
      const bool ok = trho > 1e-10;
      const double t = ok ? trho : 1.0;
      const double kf = cbrt(3.0 * pi * pi * t);
      const double ex_lda = -3.0 / (4.0 * pi) * kf;
      const double vx_lda = -kf / pi;
      const double tk2 = (t * kf) * (t * kf);
      const double den = 4.0 * kp * tk2 + mu * gg;
      const double Fx = 1.0 + kp - 4.0 * kp * kp * tk2 / den;
      if (ok) {
        ex_sum += t * ex_lda * Fx;
        vx[s] = Fx * vx_lda + 24.0 * pi * kp * kp * mu * t * t * t * gg / (den * den);
        rt = -18.0 * pi * kp * kp * mu * t * t * t * t / (den * den);
      }
      rtx[s] = rt;
    }
    // correlation (PW92 local part + PBE H)
    const double fac = ns == 2 ? 1.0 : 0.5;
    const double rhoa = rho[i] * fac, rhob = rho[(size_t)(ns - 1) * ng + i] * fac;
    const double ta = rhoa + rhob;
    const bool okc = ta > 1e-10;
    const double trho = okc ? ta : 1.0;
    double zeta = (rhoa - rhob) / trho;
    zeta = fmin(1.0, fmax(-1.0, zeta));
    const double fz = (pow(1.0 + zeta, 4.0 / 3.0) + pow(1.0 - zeta, 4.0 / 3.0) - 2.0) * const1;
    const double kf = cbrt(3.0 * pi * pi * trho);
    const double rs = cbrt(3.0 / (4.0 * pi) / trho);
    const double rssq = sqrt(rs);
    double ec_U, deU_drs, ec_P, deP_drs, alpc, dac_drs;
    pw92(0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294, rs, rssq, ec_U, deU_drs);
    pw92(0.015545, 0.20548, 1.41189e1, 6.1977, 3.3662, 0.62517, rs, rssq, ec_P, deP_drs);
    pw92(0.016887, 0.11125, 1.0357e1, 3.6231, 0.88026, 0.49671, rs, rssq, alpc, dac_drs);
    const double z4 = zeta * zeta * zeta * zeta;
    const double ec_lda = ec_U - alpc * fz * const2 * (1.0 - z4) + (ec_P - ec_U) * fz * z4;
    const double phi = 0.5 * (pow(1.0 + zeta, 2.0 / 3.0) + pow(1.0 - zeta, 2.0 / 3.0));
    const double phi3 = phi * phi * phi;
    const double T = pi * gg / (16.0 * phi * phi * kf * trho * trho);
    const double A = C1 / (exp(-ec_lda / (C2 * phi3)) - 1.0);
    const double AT = A * T;
    const double Hs = C2 * phi3 * log(1.0 + C1 * T * (1.0 + AT) / (1.0 + AT + AT * AT));
    if (okc) ec_sum += trho * (ec_lda + Hs);
    const double drs_dn = -4.0 * pi * rs * rs * rs * rs / 9.0;
    const double deU_dn = deU_drs * drs_dn, deP_dn = deP_drs * drs_dn, dac_dn = dac_drs * drs_dn;
    const double dfz_dz = 4.0 / 3.0 * (cbrt(1.0 + zeta) - cbrt(1.0 - zeta)) * const1;
    const double dec_dz = -alpc * dfz_dz * const2 * (1.0 - z4) + 4.0 * alpc * fz * const2 * zeta * zeta * zeta +
                          (ec_P - ec_U) * (dfz_dz * z4 + fz * 4.0 * zeta * zeta * zeta);
    const double dphi_dz = fabs(zeta) == 1.0 ? 0.0 : (pow(1.0 + zeta, -1.0 / 3.0) - pow(1.0 - zeta, -1.0 / 3.0)) / 3.0;
    const double tmp = 1.0 + AT + AT * AT;
    const double dH_dA = -phi3 * C1 * C2 * A * T * T * T * (2.0 + AT) / (tmp * tmp + C1 * T * (1.0 + AT) * tmp);
    const double dH_dT = phi3 * C1 * C2 * (1.0 + 2.0 * AT) / (tmp * tmp + C1 * T * (1.0 + AT) * tmp);
    const double dH_dphi = 3.0 * Hs / phi;
    const double dz_dn[2] = {2.0 * rhob / (trho * trho), -2.0 * rhoa / (trho * trho)};
    const double rtc = okc ? dH_dT * pi / (8.0 * kf * trho * phi * phi) : 0.0;
    for (int s = 0; s < ns; ++s) {
      const double dz = ns == 1 ? dz_dn[1] : dz_dn[s];
      const double dec_dn = deU_dn - dac_dn * fz * const2 * (1.0 - z4) + (deP_dn - deU_dn) * fz * z4 + dec_dz * dz;
      const double dA_dn = A * (C1 + A) / (C1 * C2 * phi3) * (dec_dn - 3.0 * ec_lda / phi * dphi_dz * dz);
      const double vc = okc ? ec_lda + Hs + trho * dec_dn + trho * dH_dA * dA_dn +
                                  dH_dT * (-7.0 / 3.0 * T - trho * 2.0 * T / phi * dphi_dz * dz) +
                                  trho * dH_dphi * dphi_dz * dz
                            : 0.0;
      vloc[(size_t)s * ng + i] = vx[s] + vc;
      const double r = rtx[s] + rtc;
      flux[((size_t)s * 3 + 0) * ng + i] = r * gxi * g.ih[0];
      flux[((size_t)s * 3 + 1) * ng + i] = r * gyi * g.ih[1];
      flux[((size_t)s * 3 + 2) * ng + i] = r * gzi * g.ih[2];
    }
  }
  xc_block_sum2(ex_sum, ec_sum, part);
}

// vxc[s] = vloc[s] - sum_a sum_m nab(m) (flux[s][a](i + m e_a) - flux[s][a](i - m e_a))
__global__ void __launch_bounds__(kXcThreads) k_xc_div(const double* __restrict__ vloc, const double* __restrict__ flux,
                                                       int ns, XcGrid g, double* __restrict__ vxc) {
  const size_t ng = (size_t)g.n1 * g.n2 * g.n3;
  for (size_t i = blockIdx.x * (size_t)kXcThreads + threadIdx.x; i < ng; i += (size_t)gridDim.x * kXcThreads) {
    const int x = (int)(i % g.n1), y = (int)((i / g.n1) % g.n2), z = (int)(i / ((size_t)g.n1 * g.n2));
    for (int s = 0; s < ns; ++s) {
      const double* fx = flux + ((size_t)s * 3 + 0) * ng;
      const double* fy = flux + ((size_t)s * 3 + 1) * ng;
      const double* fz = flux + ((size_t)s * 3 + 2) * ng;
      double dx = 0.0, dy = 0.0, dz = 0.0;
      for (int m = 1; m <= g.md; ++m) {
        dx += g.nab[m] * (fx[xc_idx(wrap(x + m, g.n1), y, z, g)] - fx[xc_idx(wrap(x - m, g.n1), y, z, g)]);
        dy += g.nab[m] * (fy[xc_idx(x, wrap(y + m, g.n2), z, g)] - fy[xc_idx(x, wrap(y - m, g.n2), z, g)]);
        dz += g.nab[m] * (fz[xc_idx(x, y, wrap(z + m, g.n3), g)] - fz[xc_idx(x, y, wrap(z - m, g.n3), g)]);
      }
      vxc[(size_t)s * ng + i] = vloc[(size_t)s * ng + i] - (dx + dy + dz);
    }
  }
}

// central FD weights of d/dx, nab(j) for j = 1..md (src/fd_module.f90:56-78)
static void nabla_coef(int md, double* nab) {
  for (int j = 1; j <= md; ++j) {
    double t = 1.0, s = 1.0;
    for (int i = -md; i <= md; ++i) {
      if (i == j) continue;
      t *= (double)(j - i);
      if (i != 0) s *= (double)(-i);
    }
    nab[j] = s / t;
  }
}

}  // namespace

extern "C" int rsdft_gpu_xc_pbe(const double* rho, double* vxc, double* exc) {
  Ctx* cp = ctx();
  RS_CHECK(cp != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");
  Ctx& c = *cp;
  RS_CHECK(rho != nullptr && vxc != nullptr, RSDFT_ERR_ARG, "xc_pbe: rho or vxc is NULL");
  const int ns = c.p.nspin;
  RS_CHECK(ns == 1 || ns == 2, RSDFT_ERR_UNSUPPORTED, "xc_pbe: nspin must be 1 or 2");
  RS_CHECK(c.p.md >= 1 && c.p.md <= kXcMdMax, RSDFT_ERR_UNSUPPORTED, "xc_pbe: Md must be 1..%d", kXcMdMax);
  const size_t ng = c.ng;
  XcGrid g{};
  g.n1 = c.p.n1;
  g.n2 = c.p.n2;
  g.n3 = c.p.n3;
  g.md = c.p.md;
  RS_CHECK(g.n1 > g.md && g.n2 > g.md && g.n3 > g.md, RSDFT_ERR_UNSUPPORTED, "xc_pbe: grid shorter than the FD order");
  for (int a = 0; a < 3; ++a) g.ih[a] = 1.0 / c.p.hgrid[a];
  nabla_coef(g.md, g.nab);
  // buffers: rho (ns), gx gy gz (3), vloc (ns), flux (3 ns), vxc (ns), partials
  const size_t nreal = ng * (size_t)(ns + 3 + ns + 3 * ns + ns);
  RS_TRY(c.scf.gga.ensure(sizeof(double) * (nreal + 2 * (size_t)kXcBlocks)));
  double* d_rho = c.scf.gga.as<double>();
  double* d_gx = d_rho + ng * ns;
  double* d_gy = d_gx + ng;
  double* d_gz = d_gy + ng;
  double* d_vl = d_gz + ng;
  double* d_fl = d_vl + ng * ns;
  double* d_v = d_fl + 3 * ng * ns;
  double* d_part = d_v + ng * ns;
  RS_CUDA(cudaMemcpyAsync(d_rho, rho, sizeof(double) * ng * ns, cudaMemcpyHostToDevice, c.stream));
  k_xc_grad<<<kXcBlocks, kXcThreads, 0, c.stream>>>(d_rho, ns, g, d_gx, d_gy, d_gz);
  k_xc_pbe<<<kXcBlocks, kXcThreads, 0, c.stream>>>(d_rho, ns, g, 0.21951, 0.804, d_gx, d_gy, d_gz, d_vl, d_fl, d_part);
  k_xc_div<<<kXcBlocks, kXcThreads, 0, c.stream>>>(d_vl, d_fl, ns, g, d_v);
  c.launches += 3;
  RS_CUDA(cudaGetLastError());
  std::vector<double> part(2 * (size_t)kXcBlocks);
  RS_CUDA(cudaMemcpyAsync(vxc, d_v, sizeof(double) * ng * ns, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaMemcpyAsync(part.data(), d_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  if (exc) {
    double ex = 0.0, ec = 0.0;
    for (int b = 0; b < kXcBlocks; ++b) {
      ex += part[2 * b];
      ec += part[2 * b + 1];
    }
    exc[0] = ex / (ns == 2 ? 2.0 : 1.0) * c.p.dv;
    exc[1] = ec * c.p.dv;
  }
  return 0;
}

}  // namespace rsdft
