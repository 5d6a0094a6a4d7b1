// Self-consistent-field pieces: density, Hartree and LDA exchange-correlation potential, the
// local-potential update and Pulay density mixing, all on the device.
//
// Reference (restated, not translated):
//   density  calc_density (src/density_module.f90): rho(:,s) = sum_{k,n} occ(n,k,s) |unk(:,n,k,s)|^2
//   Hartree  the FFT Poisson solve of calc_hartree (src/hartree/hartree_sol_fft*.f90):
//            V_H(G) = 4 pi rho(G) / |G|^2 for G != 0, V_H(G = 0) = 0; E_H = 1/2 int rho V_H
//   XC       calc_LDAPZ81 (src/xc/xc_ldapz81_module.f90): Perdew-Zunger 1981 LDA (Slater exchange,
//            Ceperley-Alder correlation fit), spin-unpolarised and polarised
//   Vloc     Vloc(:,s) = Vion + Vh + Vxc(:,s) (src/localpot_module.f90:209-215, src/scf_module.f90)
//   mixing   perform_mixing / pulay_mixing (src/mixing/mixing_module.f90:145-298,
//            src/mixing/mixing_pulay_module.f90:29-111) with IMIX = 10 (Pulay on the density,
//            the reference default), its beta search and calc_sqerr (:319-341)
//
// B200 design: the density is one pass over the resident bands per (k, s) (threads over grid
// points, bands looped inside, FP64 accumulation); the Poisson solve runs on cuFFT (D2Z / Z2D
// over the [z][y][x] grid) with one kernel for the 4 pi / G^2 factor; XC, the potential update
// and the mixing vector operations are single elementwise or reduction kernels.  The small
// Pulay system (at most MMIX = 4 unknowns) is solved on the host.
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.cuh"

namespace rsdft {
namespace {

constexpr int kScfThreads = 256;
constexpr int kScfBlocks = 4 * 148;

#define RS_CUFFT(call)                                                                             \
  do {                                                                                             \
    cufftResult r_ = (call);                                                                       \
    RS_CHECK(r_ == CUFFT_SUCCESS, RSDFT_ERR_CUDA, "%s -> cuFFT status %d", #call, (int)r_);         \
  } while (0)

// block sum of v into out[blockIdx.x] (one slot per block)
__device__ __forceinline__ void block_sum(double v, double* out) {
  __shared__ double red[kScfThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kScfThreads / 32; ++w) t += red[w];
    out[blockIdx.x] = t;
  }
}

// rho[i] += sum_n occ[n] |psi_n(i)|^2 for the nb bands of one (k, s); NC = 2: interleaved complex
template <typename T, int NC>
__global__ void __launch_bounds__(kScfThreads) k_density(const T* __restrict__ psi, const double* __restrict__ occ,
                                                         int nb, size_t ng, double* __restrict__ rho) {
  for (size_t i = blockIdx.x * (size_t)kScfThreads + threadIdx.x; i < ng; i += (size_t)gridDim.x * kScfThreads) {
    double acc = 0.0;
    for (int n = 0; n < nb; ++n) {
      const double w = occ[n];
      if (w == 0.0) continue;
      const T* p = psi + (size_t)n * ng * NC;
      if (NC == 1) {
        const double x = (double)p[i];
        acc += w * x * x;
      } else {
        const double x = (double)p[2 * i], y = (double)p[2 * i + 1];
        acc += w * (x * x + y * y);
      }
    }
    rho[i] += acc;
  }
}

// spectrum of rho (D2Z layout [n3][n2][n1/2+1]) times 4 pi / |G|^2 / ng (G = 0 term zero)
__global__ void k_poisson(cufftDoubleComplex* f, int n1, int n2, int n3, double gx, double gy, double gz, double scale) {
  const int h1 = n1 / 2 + 1;
  const long long tot = (long long)h1 * n2 * n3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
    const int i1 = (int)(t % h1);
    const int i2 = (int)((t / h1) % n2);
    const int i3 = (int)(t / ((long long)h1 * n2));
    const int m1 = i1, m2 = i2 <= n2 / 2 ? i2 : i2 - n2, m3 = i3 <= n3 / 2 ? i3 : i3 - n3;
    const double G2 = (m1 * gx) * (m1 * gx) + (m2 * gy) * (m2 * gy) + (m3 * gz) * (m3 * gz);
    const double fac = G2 > 0.0 ? 4.0 * M_PI / G2 * scale : 0.0;
    f[t].x *= fac;
    f[t].y *= fac;
  }
}

// Perdew-Zunger 1981 correlation for one spin channel set (published fit): energy per electron
// and potential for the unpolarised (u = 0) or fully polarised (u = 1) parameters.
__device__ __forceinline__ void pz81_c(double rs, int u, double& ec, double& vc) {
  const double gam[2] = {-0.1423, -0.0843}, b1[2] = {1.0529, 1.3981}, b2[2] = {0.3334, 0.2611};
  const double A[2] = {0.0311, 0.01555}, B[2] = {-0.048, -0.0269}, C[2] = {0.002, 0.0007}, D[2] = {-0.0116, -0.0048};
  if (rs >= 1.0) {
    const double sq = sqrt(rs), den = 1.0 + b1[u] * sq + b2[u] * rs;
    ec = gam[u] / den;
    vc = ec * (1.0 + (7.0 / 6.0) * b1[u] * sq + (4.0 / 3.0) * b2[u] * rs) / den;
  } else {
    const double lr = log(rs);
    ec = A[u] * lr + B[u] + C[u] * rs * lr + D[u] * rs;
    vc = A[u] * lr + (B[u] - A[u] / 3.0) + (2.0 / 3.0) * C[u] * rs * lr + ((2.0 * D[u] - C[u]) / 3.0) * rs;
  }
}

// LDA PZ81: vxc[s][i]; block partials of (sum rho exc, sum_s rho_s vxc_s)
__global__ void __launch_bounds__(kScfThreads) k_xc_pz81(const double* __restrict__ rho, size_t ng, int nspin,
                                                         double* __restrict__ vxc, double* __restrict__ part) {
  double e_sum = 0.0, v_sum = 0.0;
  const double thrpi = 3.0 / M_PI, third = 1.0 / 3.0;
  for (size_t i = blockIdx.x * (size_t)kScfThreads + threadIdx.x; i < ng; i += (size_t)gridDim.x * kScfThreads) {
    // exchange: per spin density (the factor 2^(1/3) of the polarised case) as the reference
    const double cx = nspin == 2 ? cbrt(2.0) : 1.0;
    double vx[2] = {0.0, 0.0}, ex = 0.0;
    for (int s = 0; s < nspin; ++s) {
      const double r = rho[(size_t)s * ng + i];
      if (r <= 0.0) continue;
      const double exd = -cx * 0.75 * cbrt(thrpi * r);
      ex += r * exd;
      vx[s] = (4.0 / 3.0) * exd;
    }
    // correlation: total density, spin polarisation zeta, von Barth-Hedin interpolation
    const double ra = fabs(nspin == 2 ? rho[i] : 0.5 * rho[i]);
    const double rb = fabs(nspin == 2 ? rho[ng + i] : 0.5 * rho[i]);
    const double tr = ra + rb;
    double vc[2] = {0.0, 0.0}, ec_tot = 0.0;
    if (tr > 0.0) {
      const double rs = cbrt(3.0 / (4.0 * M_PI * tr));
      double ecu, vcu, ecp, vcp;
      pz81_c(rs, 0, ecu, vcu);
      pz81_c(rs, 1, ecp, vcp);
      const double z = (ra - rb) / tr;
      const double c0 = 1.0 / (pow(2.0, 4.0 * third) - 2.0);
      const double f = (pow(1.0 + z, 4.0 * third) + pow(1.0 - z, 4.0 * third) - 2.0) * c0;
      const double dfdz = (4.0 * third) * (cbrt(1.0 + z) - cbrt(1.0 - z)) * c0;
      const double ec = ecu + f * (ecp - ecu);
      const double vcom = vcu + f * (vcp - vcu);
      const double dz = (ecp - ecu) * dfdz;
      vc[0] = vcom + dz * (1.0 - z);
      vc[1] = vcom - dz * (1.0 + z);
      ec_tot = tr * ec;
    }
    e_sum += ex + ec_tot;
    for (int s = 0; s < nspin; ++s) {
      const double v = vx[s] + vc[s];
      vxc[(size_t)s * ng + i] = v;
      v_sum += rho[(size_t)s * ng + i] * v;
    }
  }
  block_sum(e_sum, part);
  __syncthreads();
  block_sum(v_sum, part + gridDim.x);
}

// out[b] = partial sums of (a - b)(c - d) (b, d may be null: zero)
__global__ void __launch_bounds__(kScfThreads) k_dotdiff(const double* __restrict__ a, const double* __restrict__ b,
                                                         const double* __restrict__ c, const double* __restrict__ d,
                                                         size_t n, double* __restrict__ part) {
  double s = 0.0;
  for (size_t i = blockIdx.x * (size_t)kScfThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kScfThreads) {
    const double x = a[i] - (b ? b[i] : 0.0), y = c[i] - (d ? d[i] : 0.0);
    s += x * y;
  }
  block_sum(s, part);
}

// Vloc(:,s) = Vion + Vh + Vxc(:,s) in FP64 and FP32
__global__ void k_vloc(const double* __restrict__ vion, const double* __restrict__ vh, const double* __restrict__ vxc,
                       size_t ng, int nspin, double* __restrict__ v64, float* __restrict__ v32) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < ng * nspin; t += (size_t)gridDim.x * blockDim.x) {
    const size_t i = t % ng;
    const double v = vion[i] + vh[i] + vxc[t];
    v64[t] = v;
    v32[t] = (float)v;
  }
}

// Pulay combination: out = X + beta (Y - X), X = sum_i w_i Xin_i, Y = sum_i w_i Xou_i
__global__ void k_pulay_combine(const double* __restrict__ xin, const double* __restrict__ xou, const double* __restrict__ w,
                                int nw, size_t stride, size_t n, double beta, double* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    double X = 0.0, Y = 0.0;
    for (int k = 0; k < nw; ++k) {
      X += w[k] * xin[(size_t)k * stride + t];
      Y += w[k] * xou[(size_t)k * stride + t];
    }
    out[t] = X + beta * (Y - X);
  }
}

__global__ void k_scale(double* x, size_t n, double s) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) x[t] *= s;
}

// ------------------------------------------------------------------------------------------
// host helpers
// ------------------------------------------------------------------------------------------
int reduce_blocks(Ctx& c, const double* part, int nparts, std::vector<double>& out) {
  std::vector<double> h((size_t)nparts * kScfBlocks);
  RS_CUDA(cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  out.assign(nparts, 0.0);
  for (int p = 0; p < nparts; ++p)
    for (int b = 0; b < kScfBlocks; ++b) out[p] += h[(size_t)p * kScfBlocks + b];
  return 0;
}

// sum over n of (a - b)(c - d) on the device, result on the host
int dotdiff(Ctx& c, const double* a, const double* b, const double* cc, const double* d, size_t n, double& out) {
  RS_TRY(c.scf.part.ensure(sizeof(double) * 2 * kScfBlocks));
  k_dotdiff<<<kScfBlocks, kScfThreads, 0, c.stream>>>(a, b, cc, d, n, c.scf.part.as<double>());
  c.launches++;
  std::vector<double> r;
  RS_TRY(reduce_blocks(c, c.scf.part.as<double>(), 1, r));
  out = r[0];
  return 0;
}

// a device vector of ones (ng x nspin) for plain sums through k_dotdiff
const double* scf_ones(Ctx& c) {
  const size_t n = c.ng * c.p.nspin;
  if (c.scf.ones.bytes < sizeof(double) * n) {
    if (c.scf.ones.ensure(sizeof(double) * n) != 0) return nullptr;
    std::vector<double> h(n, 1.0);
    cudaMemcpy(c.scf.ones.p, h.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  }
  return c.scf.ones.as<double>();
}

int ensure_scf(Ctx& c) {
  const size_t ng = c.ng, ns = (size_t)c.p.nspin;
  RS_TRY(c.scf.vion.ensure(sizeof(double) * ng));
  RS_TRY(c.scf.rho.ensure(sizeof(double) * ng * ns));
  RS_TRY(c.scf.vh.ensure(sizeof(double) * ng));
  RS_TRY(c.scf.vxc.ensure(sizeof(double) * ng * ns));
  RS_TRY(c.vloc64.ensure(sizeof(double) * ng * ns));
  RS_TRY(c.vloc32.ensure(sizeof(float) * ng * ns));
  return 0;
}

// small dense solve A x = b (n <= 8) by Gaussian elimination with partial pivoting
bool small_solve(std::vector<double> A, std::vector<double>& b, int n) {
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < n; ++j) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      const double f = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; ++j) A[i * n + j] -= f * A[k * n + j];
      b[i] -= f * b[k];
    }
  }
  for (int k = n - 1; k >= 0; --k) {
    double s = b[k];
    for (int j = k + 1; j < n; ++j) s -= A[k * n + j] * b[j];
    b[k] = s / A[k * n + k];
  }
  return true;
}

}  // namespace
}  // namespace rsdft

using namespace rsdft;

#define SCF_CTX()                                                                   \
  Ctx* cp_ = ctx();                                                                 \
  RS_CHECK(cp_ != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");   \
  Ctx& c = *cp_

extern "C" int rsdft_gpu_set_vion(const double* vion, int ml) {
  SCF_CTX();
  RS_CHECK(vion != nullptr && (size_t)ml == c.ng, RSDFT_ERR_ARG, "set_vion: bad arguments");
  for (size_t i = 0; i < c.ng; ++i) RS_CHECK(std::isfinite(vion[i]), RSDFT_ERR_NUMERIC, "Vion(%zu) is not finite", i + 1);
  RS_TRY(ensure_scf(c));
  RS_CUDA(cudaMemcpy(c.scf.vion.p, vion, sizeof(double) * c.ng, cudaMemcpyHostToDevice));
  return 0;
}

extern "C" int rsdft_gpu_set_rho(const double* rho, int ml) {
  SCF_CTX();
  RS_CHECK(rho != nullptr && (size_t)ml == c.ng, RSDFT_ERR_ARG, "set_rho: bad arguments");
  RS_TRY(ensure_scf(c));
  RS_CUDA(cudaMemcpy(c.scf.rho.p, rho, sizeof(double) * c.ng * c.p.nspin, cudaMemcpyHostToDevice));
  c.scf.have_rho = true;
  return 0;
}

extern "C" int rsdft_gpu_get_rho(double* rho, double* vh, double* vxc) {
  SCF_CTX();
  RS_CHECK(c.scf.have_rho, RSDFT_ERR_STATE, "no density on the device");
  const size_t ns = (size_t)c.p.nspin;
  RS_CUDA(cudaStreamSynchronize(c.stream));
  if (rho) RS_CUDA(cudaMemcpy(rho, c.scf.rho.p, sizeof(double) * c.ng * ns, cudaMemcpyDeviceToHost));
  if (vh) RS_CUDA(cudaMemcpy(vh, c.scf.vh.p, sizeof(double) * c.ng, cudaMemcpyDeviceToHost));
  if (vxc) RS_CUDA(cudaMemcpy(vxc, c.scf.vxc.p, sizeof(double) * c.ng * ns, cudaMemcpyDeviceToHost));
  return 0;
}

extern "C" int rsdft_gpu_density(const double* occ) {
  SCF_CTX();
  RS_CHECK(occ != nullptr, RSDFT_ERR_ARG, "density: occ is NULL");
  RS_TRY(ensure_scf(c));
  const int mb = c.p.mb, nk = c.p.nk, ns = c.p.nspin;
  RS_CUDA(cudaMemsetAsync(c.scf.rho.p, 0, sizeof(double) * c.ng * ns, c.stream));
  RS_TRY(c.scf.occ.ensure(sizeof(double) * (size_t)mb * nk * ns));
  RS_CUDA(cudaMemcpyAsync(c.scf.occ.p, occ, sizeof(double) * (size_t)mb * nk * ns, cudaMemcpyHostToDevice, c.stream));
  ProfScope ps(c, "density");
  for (int s = 0; s < ns; ++s)
    for (int k = 0; k < nk; ++k) {
      WaveFns& w = c.wfn(k, s);
      RS_CHECK(w.valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k + 1, s + 1);
      const double* o = c.scf.occ.as<double>() + ((size_t)s * nk + k) * mb;
      double* r = c.scf.rho.as<double>() + (size_t)s * c.ng;
      const int nb = c.kp[k].nband;
      if (c.cplx) {
        if (c.mixed) k_density<float, 2><<<kScfBlocks, kScfThreads, 0, c.stream>>>(w.psi.as<float>(), o, nb, c.ng, r);
        else k_density<double, 2><<<kScfBlocks, kScfThreads, 0, c.stream>>>(w.psi.as<double>(), o, nb, c.ng, r);
      } else {
        if (c.mixed) k_density<float, 1><<<kScfBlocks, kScfThreads, 0, c.stream>>>(w.psi.as<float>(), o, nb, c.ng, r);
        else k_density<double, 1><<<kScfBlocks, kScfThreads, 0, c.stream>>>(w.psi.as<double>(), o, nb, c.ng, r);
      }
      c.launches++;
    }
  c.scf.have_rho = true;
  return check_launch("density");
}

extern "C" int rsdft_gpu_normalize_density(double nelec) {
  SCF_CTX();
  RS_CHECK(c.scf.have_rho && nelec > 0.0, RSDFT_ERR_STATE, "normalize_density: no density");
  const size_t n = c.ng * c.p.nspin;
  double q = 0.0;
  RS_CHECK(scf_ones(c) != nullptr, RSDFT_ERR_OOM, "normalize_density: no memory");
  RS_TRY(dotdiff(c, c.scf.rho.as<double>(), nullptr, scf_ones(c), nullptr, n, q));
  q *= c.p.dv;
  RS_CHECK(q > 0.0, RSDFT_ERR_NUMERIC, "normalize_density: charge %g", q);
  k_scale<<<kScfBlocks, kScfThreads, 0, c.stream>>>(c.scf.rho.as<double>(), n, nelec / q);
  c.launches++;
  return check_launch("normalize_density");
}

// ene[0] E_H = 1/2 int rho V_H, ene[1] E_xc, ene[2] int rho V_xc, ene[3] total charge
extern "C" int rsdft_gpu_potential(double* ene) {
  SCF_CTX();
  RS_CHECK(c.scf.have_rho, RSDFT_ERR_STATE, "potential: no density on the device");
  RS_CHECK(c.scf.vion.p != nullptr, RSDFT_ERR_STATE, "potential: rsdft_gpu_set_vion has not been called");
  RS_TRY(ensure_scf(c));
  const int n1 = c.p.n1, n2 = c.p.n2, n3 = c.p.n3, ns = c.p.nspin;
  const size_t ng = c.ng, nh = (size_t)(n1 / 2 + 1) * n2 * n3;
  ProfScope ps(c, "potential");
  // total density -> Hartree
  RS_TRY(c.scf.work.ensure(sizeof(double) * ng + sizeof(cufftDoubleComplex) * nh));
  double* rt = c.scf.work.as<double>();
  cufftDoubleComplex* spec = reinterpret_cast<cufftDoubleComplex*>(rt + ng);
  RS_CUDA(cudaMemcpyAsync(rt, c.scf.rho.p, sizeof(double) * ng, cudaMemcpyDeviceToDevice, c.stream));
  if (ns == 2) {
    RS_TRY(c.scf.part.ensure(sizeof(double) * 2 * kScfBlocks));
    cublasHandle_t h = c.cublas;
    const double one = 1.0;
    cublasSetStream(h, c.stream);
    RS_CHECK(cublasDaxpy(h, (int)ng, &one, c.scf.rho.as<double>() + ng, 1, rt, 1) == CUBLAS_STATUS_SUCCESS,
             RSDFT_ERR_CUDA, "daxpy failed");
  }
  if (!c.scf.plans) {
    RS_CUFFT(cufftPlan3d(&c.scf.plan_f, n3, n2, n1, CUFFT_D2Z));
    RS_CUFFT(cufftPlan3d(&c.scf.plan_b, n3, n2, n1, CUFFT_Z2D));
    c.scf.plans = true;
  }
  RS_CUFFT(cufftSetStream(c.scf.plan_f, c.stream));
  RS_CUFFT(cufftSetStream(c.scf.plan_b, c.stream));
  RS_CUFFT(cufftExecD2Z(c.scf.plan_f, rt, spec));
  const double L1 = n1 * c.p.hgrid[0], L2 = n2 * c.p.hgrid[1], L3 = n3 * c.p.hgrid[2];
  k_poisson<<<kScfBlocks, kScfThreads, 0, c.stream>>>(spec, n1, n2, n3, 2.0 * M_PI / L1, 2.0 * M_PI / L2,
                                                      2.0 * M_PI / L3, 1.0 / (double)ng);
  c.launches++;
  RS_CUFFT(cufftExecZ2D(c.scf.plan_b, spec, c.scf.vh.as<double>()));
  // XC
  RS_TRY(c.scf.part.ensure(sizeof(double) * 2 * kScfBlocks));
  k_xc_pz81<<<kScfBlocks, kScfThreads, 0, c.stream>>>(c.scf.rho.as<double>(), ng, ns, c.scf.vxc.as<double>(),
                                                      c.scf.part.as<double>());
  c.launches++;
  std::vector<double> xc;
  RS_TRY(reduce_blocks(c, c.scf.part.as<double>(), 2, xc));
  double eh = 0.0, q = 0.0;
  RS_TRY(dotdiff(c, rt, nullptr, c.scf.vh.as<double>(), nullptr, ng, eh));
  RS_CHECK(scf_ones(c) != nullptr, RSDFT_ERR_OOM, "potential: no memory");
  RS_TRY(dotdiff(c, rt, nullptr, scf_ones(c), nullptr, ng, q));
  // Vloc = Vion + Vh + Vxc
  k_vloc<<<kScfBlocks, kScfThreads, 0, c.stream>>>(c.scf.vion.as<double>(), c.scf.vh.as<double>(),
                                                   c.scf.vxc.as<double>(), ng, ns, c.vloc64.as<double>(),
                                                   c.vloc32.as<float>());
  c.launches++;
  RS_TRY(check_launch("potential"));
  if (ene) {
    ene[0] = 0.5 * eh * c.p.dv;
    ene[1] = xc[0] * c.p.dv;
    ene[2] = xc[1] * c.p.dv;
    ene[3] = q * c.p.dv;
  }
  for (int s = 0; s < ns; ++s) c.vloc_set[s] = true;
  return 0;
}

extern "C" int rsdft_gpu_init_mixing(int mmix, double beta) {
  SCF_CTX();
  RS_CHECK(mmix >= 1 && mmix <= 8 && beta > 0.0, RSDFT_ERR_ARG, "init_mixing: mmix 1..8, beta > 0");
  RS_CHECK(c.scf.have_rho && c.vloc_set[0], RSDFT_ERR_STATE, "init_mixing: density and potential must be set first");
  const size_t n = c.ng * c.p.nspin;
  auto& m = c.scf;
  m.mmix = mmix;
  m.beta = beta;
  m.mmix_count = 0;
  m.dif0 = 0.0;
  RS_TRY(m.xin.ensure(sizeof(double) * n * mmix));
  RS_TRY(m.xou.ensure(sizeof(double) * n * mmix));
  RS_TRY(m.xin_bak.ensure(sizeof(double) * n * mmix));
  RS_TRY(m.xou_bak.ensure(sizeof(double) * n * mmix));
  RS_TRY(m.xold_f.ensure(sizeof(double) * n));
  RS_TRY(m.xold_g.ensure(sizeof(double) * n));
  RS_TRY(m.h.ensure(sizeof(double) * n));
  RS_CUDA(cudaMemsetAsync(m.xin.p, 0, sizeof(double) * n * mmix, c.stream));
  RS_CUDA(cudaMemsetAsync(m.xou.p, 0, sizeof(double) * n * mmix, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xold_f.p, m.rho.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xold_g.p, c.vloc64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xin.as<double>() + (size_t)(mmix - 1) * n, m.rho.p, sizeof(double) * n,
                          cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  m.mixing = true;
  return 0;
}

// calc_sqerr: sqerr[s] = sum (Vloc_s - Xold_g,s)^2 / ML, sqerr[nspin + s] = sum (rho_s - Xold_f,s)^2 / ML
extern "C" int rsdft_gpu_sqerr(double* sqerr) {
  SCF_CTX();
  RS_CHECK(c.scf.mixing && sqerr, RSDFT_ERR_STATE, "sqerr: rsdft_gpu_init_mixing has not been called");
  const size_t ng = c.ng;
  for (int s = 0; s < c.p.nspin; ++s) {
    const double* v = c.vloc64.as<double>() + s * ng;
    const double* g = c.scf.xold_g.as<double>() + s * ng;
    const double* r = c.scf.rho.as<double>() + s * ng;
    const double* f = c.scf.xold_f.as<double>() + s * ng;
    double a = 0.0, b = 0.0;
    RS_TRY(dotdiff(c, v, g, v, g, ng, a));
    RS_TRY(dotdiff(c, r, f, r, f, ng, b));
    sqerr[s] = a / (double)ng;
    sqerr[c.p.nspin + s] = b / (double)ng;
  }
  return 0;
}

// one pulay_mixing call (src/mixing/mixing_pulay_module.f90:29-111) on h with history Xin / Xou
static int pulay_step(Ctx& c, double beta) {
  auto& m = c.scf;
  const size_t n = c.ng * c.p.nspin;
  const int mm = m.mmix;
  double* xin = m.xin.as<double>();
  double* xou = m.xou.as<double>();
  RS_CUDA(cudaMemcpyAsync(xou + (size_t)(mm - 1) * n, m.h.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  m.mmix_count++;
  const int m0 = std::min(m.mmix_count, mm);
  if (mm == 1 || m0 < mm) {  // simple mixing while the history fills
    for (int i = 1; i < mm; ++i) {
      RS_CUDA(cudaMemcpyAsync(xin + (size_t)(i - 1) * n, xin + (size_t)i * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
      RS_CUDA(cudaMemcpyAsync(xou + (size_t)(i - 1) * n, xou + (size_t)i * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
    }
    // Xin(mmix) = Xin(mmix) + beta (Xou(mmix) - Xin(mmix)); h = Xin(mmix)
    std::vector<double> w = {1.0};
    RS_TRY(m.w.ensure(sizeof(double) * 8));
    RS_CUDA(cudaMemcpyAsync(m.w.p, w.data(), sizeof(double), cudaMemcpyHostToDevice, c.stream));
    k_pulay_combine<<<kScfBlocks, kScfThreads, 0, c.stream>>>(xin + (size_t)(mm - 1) * n, xou + (size_t)(mm - 1) * n,
                                                              m.w.as<double>(), 1, n, n, beta, m.h.as<double>());
    c.launches++;
    RS_CUDA(cudaMemcpyAsync(xin + (size_t)(mm - 1) * n, m.h.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return check_launch("mixing");
  }
  std::vector<double> A((size_t)m0 * m0), b((size_t)m0, 1.0);
  for (int j0 = 0; j0 < m0; ++j0)
    for (int i0 = j0; i0 < m0; ++i0) {
      const int i = mm - m0 + i0, j = mm - m0 + j0;
      double v = 0.0;
      RS_TRY(dotdiff(c, xou + (size_t)i * n, xin + (size_t)i * n, xou + (size_t)j * n, xin + (size_t)j * n, n, v));
      A[(size_t)i0 * m0 + j0] = v;
      A[(size_t)j0 * m0 + i0] = v;
    }
  RS_CHECK(small_solve(A, b, m0), RSDFT_ERR_NUMERIC, "Pulay mixing: singular residual overlap");
  double sb = 0.0;
  for (double x : b) sb += x;
  for (double& x : b) x /= sb;
  RS_TRY(m.w.ensure(sizeof(double) * 8));
  RS_CUDA(cudaMemcpyAsync(m.w.p, b.data(), sizeof(double) * m0, cudaMemcpyHostToDevice, c.stream));
  k_pulay_combine<<<kScfBlocks, kScfThreads, 0, c.stream>>>(xin + (size_t)(mm - m0) * n, xou + (size_t)(mm - m0) * n,
                                                            m.w.as<double>(), m0, n, n, beta, m.h.as<double>());
  c.launches++;
  for (int i = std::max(1, mm - m0); i <= mm - 1; ++i) {
    RS_CUDA(cudaMemcpyAsync(xin + (size_t)(i - 1) * n, xin + (size_t)i * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
    RS_CUDA(cudaMemcpyAsync(xou + (size_t)(i - 1) * n, xou + (size_t)i * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  }
  RS_CUDA(cudaMemcpyAsync(xin + (size_t)(mm - 1) * n, m.h.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return check_launch("mixing");
}

// perform_mixing with IMIX = 10: Pulay on the density, the beta search for beta > 1
// (src/mixing/mixing_module.f90:145-298); on return the device density is the mixed one and
// Xold holds (mixed density, the potential of the unmixed density).
extern "C" int rsdft_gpu_mix_density(double* beta_used) {
  SCF_CTX();
  auto& m = c.scf;
  RS_CHECK(m.mixing, RSDFT_ERR_STATE, "mix_density: rsdft_gpu_init_mixing has not been called");
  const size_t n = c.ng * c.p.nspin;
  const size_t bytes_hist = sizeof(double) * n * m.mmix;
  ProfScope ps(c, "mixing");
  // h = f (the density); keep the history to restart a rejected trial
  RS_CUDA(cudaMemcpyAsync(m.h.p, m.rho.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_TRY(m.f0.ensure(sizeof(double) * n));
  RS_CUDA(cudaMemcpyAsync(m.f0.p, m.rho.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xin_bak.p, m.xin.p, bytes_hist, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xou_bak.p, m.xou.p, bytes_hist, cudaMemcpyDeviceToDevice, c.stream));
  const int count_bak = m.mmix_count;
  double beta = m.beta, beta_min = beta, dif_min = 1e10;
  int max_loop = 1;
  if (beta > 1.0) {
    if (m.dif0 == 0.0) {
      max_loop = 1;
      beta = 0.05;
    } else {
      max_loop = 11;
      beta = 1.0;
    }
  }
  double dif1 = 0.0;
  for (int loop = 1; loop <= max_loop; ++loop) {
    RS_TRY(pulay_step(c, beta));
    RS_TRY(dotdiff(c, m.h.as<double>(), m.xold_f.as<double>(), m.h.as<double>(), m.xold_f.as<double>(), n, dif1));
    dif1 /= (double)c.ng;
    const double diff = m.dif0 != 0.0 ? dif1 / m.dif0 : 0.0;
    if (dif1 < dif_min) {
      beta_min = beta;
      dif_min = dif1;
    }
    if (loop < max_loop) {
      if (diff > 0.5) {
        RS_CUDA(cudaMemcpyAsync(m.xin.p, m.xin_bak.p, bytes_hist, cudaMemcpyDeviceToDevice, c.stream));
        RS_CUDA(cudaMemcpyAsync(m.xou.p, m.xou_bak.p, bytes_hist, cudaMemcpyDeviceToDevice, c.stream));
        RS_CUDA(cudaMemcpyAsync(m.h.p, m.f0.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
        m.mmix_count = count_bak;
        beta *= 0.5;
      } else {
        break;
      }
      if (loop == max_loop - 1) beta = beta_min;
    }
  }
  if (beta_used) *beta_used = beta;
  m.dif0 = dif1;
  // f = h (mixed density); Xold = (f, g = the potential of the unmixed density)
  RS_CUDA(cudaMemcpyAsync(m.rho.p, m.h.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xold_f.p, m.h.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaMemcpyAsync(m.xold_g.p, c.vloc64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

namespace rsdft {
void scf_release(Ctx& c) {
  auto& m = c.scf;
  if (m.plans) {
    cufftDestroy(m.plan_f);
    cufftDestroy(m.plan_b);
    m.plans = false;
  }
  DBuf* bufs[] = {&m.vion, &m.rho, &m.vh, &m.vxc, &m.occ, &m.work, &m.part, &m.ones, &m.xin, &m.xou,
                  &m.xin_bak, &m.xou_bak, &m.xold_f, &m.xold_g, &m.h, &m.f0, &m.w, &m.gga};
  for (DBuf* b : bufs) b->release();
  m.have_rho = m.mixing = false;
}
}  // namespace rsdft
