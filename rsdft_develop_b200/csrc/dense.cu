// Dense band-space operations: Gram-Schmidt (Cholesky QR) and subspace diagonalisation.
//
// Reference semantics:
//   gram_schmidt_t (src/gram_schmidt/gram_schmidt_t_module.f90:85-308) orthonormalises the
//   bands in order with the dV inner product; its result is the Q factor of Psi = Q R with
//   R upper triangular and positive diagonal.  Cholesky QR (the reference's GS=4 variant,
//   src/gram_schmidt/gram_schmidt_lusl_module.f90:241-328: S = dV Psi^H Psi, potrf, trtri,
//   Psi <- Psi R^-1) produces the same Q, with O(N M^2) GEMM work instead of a recursion.
//   subspace_diag_la (src/subspace_diag/subspace_diag_la_module.f90:18-223):
//   Hsub = 1/2 dV (Psi^H H Psi + (H Psi)^H Psi) (dsyr2k / zher2k), dsyev / zheevd, Psi <- Psi V.
// FP64 path: cuBLAS syrk/herk, syr2k/her2k, trsm, gemm and cuSOLVER potrf, syevd/heevd.
// Mixed mode keeps psi in FP32; the split-BF16 tensor-core contractions live in gemm_x3.cu.
// Inside the sweep the two steps run fused as one Cholesky-Rayleigh-Ritz step (gssd_run).
#include <cstring>

#include "ctx.cuh"

namespace rsdft {

#define RS_CUBLAS(call)                                                                  \
  do {                                                                                   \
    cublasStatus_t st_ = (call);                                                         \
    if (st_ != CUBLAS_STATUS_SUCCESS) {                                                  \
      set_error(RSDFT_ERR_CUDA, "%s:%d %s -> cuBLAS status %d", __FILE__, __LINE__, #call, \
                (int)st_);                                                               \
      return RSDFT_ERR_CUDA;                                                             \
    }                                                                                    \
  } while (0)
#define RS_CUSOLVER(call)                                                                   \
  do {                                                                                      \
    cusolverStatus_t st_ = (call);                                                          \
    if (st_ != CUSOLVER_STATUS_SUCCESS) {                                                   \
      set_error(RSDFT_ERR_CUDA, "%s:%d %s -> cuSOLVER status %d", __FILE__, __LINE__, #call, \
                (int)st_);                                                                  \
      return RSDFT_ERR_CUDA;                                                                \
    }                                                                                       \
  } while (0)

// FP64 view of the resident wavefunctions (mixed mode converts through a workspace).
struct F64View {
  double* x = nullptr;
  bool converted = false;
};

static size_t nreal(const Ctx& c) { return c.ng * (c.cplx ? 2 : 1); }

static int f64_view(Ctx& c, int k, int s, F64View& v) {
  const int nb = c.kp[k].nband;
  if (!c.mixed) {
    v.x = c.wfn(k, s).psi.as<double>();
    return 0;
  }
  RS_TRY(c.ws_f64.ensure(sizeof(double) * nreal(c) * nb));
  RS_TRY(convert_f2d(c, c.wfn(k, s).psi.as<float>(), c.ws_f64.as<double>(), nreal(c) * nb));
  v.x = c.ws_f64.as<double>();
  v.converted = true;
  return 0;
}
static int f64_commit(Ctx& c, int k, int s, F64View& v) {
  if (!v.converted) return 0;
  return convert_d2f(c, v.x, c.wfn(k, s).psi.as<float>(), nreal(c) * c.kp[k].nband);
}

static int read_info(Ctx& c, int* d_info, int* h_info) {
  RS_CUDA(cudaMemcpyAsync(h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

// ---------------------------------------------------------------------------
// FP64 Gram matrices of a few bands (nb <= 44): cuBLAS syrk/syrkx/syr2k pick slow kernels for
// an nb x nb result over a long grid (O2 sample: 3.4 ms per call at nb = 18, ng = 48^3), so the
// real build forms them here.  Upper triangles (i <= j, column-major) of
//   S = dV X^T X,  M = dV X^T (H X)  or  M = dV/2 (X^T (H X) + (H X)^T X),
// each CTA summing a contiguous range of grid points into per-CTA partials, then a fixed-order
// reduction (deterministic).
// ---------------------------------------------------------------------------
constexpr int kGramTK = 64;     // grid points per shared-memory tile
constexpr int kGramPmax = 4;    // pairs per thread (256 threads: npair <= 1024, nb <= 44)
constexpr int kGramNbMax = 44;

__global__ void __launch_bounds__(256) k_gram_small(const double* __restrict__ X, const double* __restrict__ HX,
                                                    int ng, int nb, int npair, int mode, int kper,
                                                    double* __restrict__ part) {
  extern __shared__ double gsm[];
  double* sx = gsm;                       // [kGramTK][nb]
  double* sh = gsm + kGramTK * nb;        // [kGramTK][nb]
  const bool wantS = mode & 1, wantM = mode & 2, sym = mode & 4;
  int pi[kGramPmax], pj[kGramPmax];
  double aS[kGramPmax], aM[kGramPmax];
#pragma unroll
  for (int q = 0; q < kGramPmax; ++q) {
    const int p = threadIdx.x + q * 256;
    int j = 0;
    while ((j + 1) * (j + 2) / 2 <= p) ++j;   // p = j (j + 1) / 2 + i, i <= j
    pj[q] = j;
    pi[q] = p - j * (j + 1) / 2;
    aS[q] = 0.0;
    aM[q] = 0.0;
  }
  const int k0 = blockIdx.x * kper, k1 = min(ng, k0 + kper);
  for (int kk = k0; kk < k1; kk += kGramTK) {
    const int tk = min(kGramTK, k1 - kk);
    for (int idx = threadIdx.x; idx < tk * nb; idx += 256) {
      const int b = idx / tk, t = idx - b * tk;
      sx[t * nb + b] = X[(size_t)b * ng + kk + t];
      if (wantM) sh[t * nb + b] = HX[(size_t)b * ng + kk + t];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kGramPmax; ++q) {
      if (threadIdx.x + q * 256 >= npair) break;
      const int i = pi[q], j = pj[q];
      double s0 = 0.0, m0 = 0.0;
      for (int t = 0; t < tk; ++t) {
        const double xi = sx[t * nb + i], xj = sx[t * nb + j];
        if (wantS) s0 += xi * xj;
        if (wantM) m0 += sym ? xi * sh[t * nb + j] + sh[t * nb + i] * xj : xi * sh[t * nb + j];
      }
      aS[q] += s0;
      aM[q] += m0;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < kGramPmax; ++q) {
    const int p = threadIdx.x + q * 256;
    if (p >= npair) break;
    part[((size_t)blockIdx.x * 2 + 0) * npair + p] = aS[q];
    part[((size_t)blockIdx.x * 2 + 1) * npair + p] = aM[q];
  }
}

__global__ void k_gram_small_reduce(const double* __restrict__ part, int nblk, int npair, int nb, int mode,
                                    double sS, double sM, double* __restrict__ S, double* __restrict__ M) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npair) return;
  int j = 0;
  while ((j + 1) * (j + 2) / 2 <= p) ++j;
  const int i = p - j * (j + 1) / 2;
  double ts = 0.0, tm = 0.0;
  for (int b = 0; b < nblk; ++b) {
    ts += part[((size_t)b * 2 + 0) * npair + p];
    tm += part[((size_t)b * 2 + 1) * npair + p];
  }
  if (mode & 1) S[i + (size_t)j * nb] = sS * ts;
  if (mode & 2) M[i + (size_t)j * nb] = sM * tm;
}

// S (if non-null) = dV X^T X, M (if non-null) = dV X^T HX or, sym, dV/2 (X^T HX + HX^T X):
// upper triangles; the lower triangles are left as they were
static int gram_small_f64(Ctx& c, const double* X, const double* HX, int ng, int nb, double dV, double* S, double* M,
                          bool sym) {
  const int npair = nb * (nb + 1) / 2;
  const int mode = (S ? 1 : 0) | (M ? 2 : 0) | (sym ? 4 : 0);
  int nblk = std::min(2 * 148, std::max(1, (ng + kGramTK - 1) / kGramTK));
  int kper = (ng + nblk - 1) / nblk;
  kper = (kper + kGramTK - 1) / kGramTK * kGramTK;
  nblk = (ng + kper - 1) / kper;
  RS_TRY(c.ws_gram.ensure(sizeof(double) * 2 * (size_t)npair * nblk));
  const size_t smem = sizeof(double) * 2 * kGramTK * nb;
  k_gram_small<<<nblk, 256, smem, c.stream>>>(X, HX, ng, nb, npair, mode, kper, c.ws_gram.as<double>());
  k_gram_small_reduce<<<(npair + 127) / 128, 128, 0, c.stream>>>(c.ws_gram.as<double>(), nblk, npair, nb, mode, dV,
                                                                  sym ? 0.5 * dV : dV, S, M);
  c.launches += 2;
  RS_CUDA(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// mixed precision (real8): psi stays FP32; S, Hsub and the rotations run as split-BF16
// tensor-core GEMMs with FP64 results; Cholesky, R^-1 and the eigensolve stay FP64.
// ---------------------------------------------------------------------------
__global__ void k_symmetrize(double* H, int n) {
  // H <- (H + H^T)/2, full matrix, column-major
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    if (i < j) {
      const double a = 0.5 * (H[i + (long long)j * n] + H[j + (long long)i * n]);
      H[i + (long long)j * n] = a;
      H[j + (long long)i * n] = a;
    }
  }
}
__global__ void k_fill_lower(double* H, int n) {
  // H(i, j) <- H(j, i) for i > j (column-major): the lower triangle from the upper
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    if (i > j) H[i + (long long)j * n] = H[j + (long long)i * n];
  }
}
// Rotation in update form: each column j of C = R^-1 V (an eigenvector, defined up to sign)
// is signed so that C(j, j) >= 0, then C <- C - I.  Near convergence C is close to I, so the
// rotation X (I + D) = X + X D forms a small correction.
__global__ void k_rotation_update_form(double* C, int n) {
  const int j = blockIdx.x;
  if (j >= n) return;
  double* col = C + (long long)j * n;
  const double sg = col[j] < 0.0 ? -1.0 : 1.0;
  __syncthreads();  // every thread has read C(j, j) before any thread writes the column
  for (int i = threadIdx.x; i < n; i += blockDim.x) col[i] = sg * col[i] - (i == j ? 1.0 : 0.0);
}
__global__ void k_identity(double* I, int n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x)
    I[t] = (t % n) == (t / n) ? 1.0 : 0.0;
}

// Eigen-decomposition of the nb x nb Hermitian matrix in H (upper triangle, column-major):
// eigenvalues ascending into W, eigenvectors overwrite H.  FP64 cuSOLVER: divide and conquer
// (syevd/heevd, the reference's dsyev/zheevd role) or Jacobi (syevj/heevj), chosen at init.
static int eig_solve(Ctx& c, int nb, void* H, double* W) {
  ProfScope ps(c, "sd_eig");
  int lwork = 0, info = 0;
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  if (c.eig_jacobi) {
    if (!c.syevj) {
      RS_CUSOLVER(cusolverDnCreateSyevjInfo(&c.syevj));
      RS_CUSOLVER(cusolverDnXsyevjSetTolerance(c.syevj, 1.0e-15));
      RS_CUSOLVER(cusolverDnXsyevjSetMaxSweeps(c.syevj, 30));
    }
    if (c.cplx) {
      RS_CUSOLVER(cusolverDnZheevj_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                                              (cuDoubleComplex*)H, nb, W, &lwork, c.syevj));
      RS_TRY(c.ws_solver.ensure(sizeof(cuDoubleComplex) * (size_t)std::max(lwork, 1)));
      RS_CUSOLVER(cusolverDnZheevj(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                                   (cuDoubleComplex*)H, nb, W, c.ws_solver.as<cuDoubleComplex>(), lwork,
                                   c.ws_info.as<int>(), c.syevj));
    } else {
      RS_CUSOLVER(cusolverDnDsyevj_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                                              (double*)H, nb, W, &lwork, c.syevj));
      RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
      RS_CUSOLVER(cusolverDnDsyevj(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, (double*)H, nb, W,
                                   c.ws_solver.as<double>(), lwork, c.ws_info.as<int>(), c.syevj));
    }
  } else if (c.cplx) {
    RS_CUSOLVER(cusolverDnZheevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb,
                                            (cuDoubleComplex*)H, nb, W, &lwork));
    RS_TRY(c.ws_solver.ensure(sizeof(cuDoubleComplex) * (size_t)std::max(lwork, 1)));
    RS_CUSOLVER(cusolverDnZheevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, (cuDoubleComplex*)H,
                                 nb, W, c.ws_solver.as<cuDoubleComplex>(), lwork, c.ws_info.as<int>()));
  } else {
    RS_CUSOLVER(cusolverDnDsyevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, (double*)H,
                                            nb, W, &lwork));
    RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
    RS_CUSOLVER(cusolverDnDsyevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, (double*)H, nb, W,
                                 c.ws_solver.as<double>(), lwork, c.ws_info.as<int>()));
  }
  RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
  RS_CHECK(info == 0, RSDFT_ERR_EIG, "subspace eigensolver failed (info=%d)", info);
  return 0;
}

static int gs_mixed_real(Ctx& c, int k, int s, int passes) {
  const int nb = c.kp[k].nband;
  float* X = c.wfn(k, s).psi.as<float>();
  RS_TRY(c.ws_dense.ensure(sizeof(double) * 2 * (size_t)nb * nb));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* S = c.ws_dense.as<double>();
  double* Ri = S + (size_t)nb * nb;
  int lwork = 0;
  RS_CUSOLVER(cusolverDnDpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, &lwork));
  RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
  const double one = 1.0;
  for (int pass = 0; pass < std::max(1, passes); ++pass) {
    RS_CUDA(cudaMemsetAsync(S, 0, sizeof(double) * (size_t)nb * nb, c.stream));
    // S[m][n] = dV sum_g X[m][g] X[n][g] (symmetric, row/column major alike)
    RS_TRY(gemm_tn_x3(c, X, (long long)c.ng, nb, X, (long long)c.ng, nb, (long long)c.ng, c.p.dv, S, nb, 0,
                      c.gemm_terms_sm));
    {
      ProfScope ps(c, "gs");
      RS_CUSOLVER(cusolverDnDpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<double>(), lwork,
                                   c.ws_info.as<int>()));
      int info = 0;
      RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
      RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (potrf info=%d)", info);
      k_identity<<<64, 256, 0, c.stream>>>(Ri, nb);
      c.launches++;
      RS_CUBLAS(cublasDtrsm(c.cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nb,
                            nb, &one, S, nb, Ri, nb));
    }
    // X <- X R^-1
    RS_TRY(gemm_rotate_x3(c, X, (long long)c.ng, nb, (long long)c.ng, Ri, nb, c.gemm_terms_rot));
  }
  return 0;
}

static int sd_mixed_real(Ctx& c, int k, int s, double* h_esp) {
  const int nb = c.kp[k].nband;
  float* X = c.wfn(k, s).psi.as<float>();
  RS_TRY(c.ws_hpsi.ensure(sizeof(float) * c.ng * nb));
  float* HX = c.ws_hpsi.as<float>();
  RS_TRY(hpsi_real<float>(c, k, s, X, HX, c.ng, nb));
  RS_TRY(c.ws_dense.ensure(sizeof(double) * ((size_t)nb * nb + nb)));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* H = c.ws_dense.as<double>();
  double* W = H + (size_t)nb * nb;
  RS_CUDA(cudaMemsetAsync(H, 0, sizeof(double) * (size_t)nb * nb, c.stream));
  // H[m][n] = dV sum_g X[m][g] (HX)[n][g]; Hsub = (H + H^T)/2 = 1/2 dV (X^T HX + HX^T X)
  RS_TRY(gemm_tn_x3(c, X, (long long)c.ng, nb, HX, (long long)c.ng, nb, (long long)c.ng, c.p.dv, H, nb, 0,
                      c.gemm_terms_sm));
  k_symmetrize<<<64, 256, 0, c.stream>>>(H, nb);
  c.launches++;
  RS_TRY(eig_solve(c, nb, H, W));
  RS_TRY(gemm_rotate_x3(c, X, (long long)c.ng, nb, (long long)c.ng, H, nb, c.gemm_terms_rot));
  if (h_esp) {
    RS_CUDA(cudaMemcpyAsync(h_esp, W, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return 0;
}

// ---------------------------------------------------------------------------
// mixed precision (complex16): psi stays FP32 (interleaved); the complex overlaps are real
// split-BF16 contractions over the interleaved view, Re(conj(a) b) = x_a . x_b and
// Im(conj(a) b) = x_a . J x_b with J (re, im) = (im, -re); the rotation by a complex matrix is
// the real rotation of the (re, im) pairs by its 2 nb x 2 nb real form (gemm_x3.cu).  Cholesky,
// R^-1 and the eigensolve stay FP64 (zpotrf, ztrsm, zheevd).
// ---------------------------------------------------------------------------
// Z(i, j) (column-major complex) = Re[i][j] + i Im[i][j] (row-major real parts)
__global__ void k_assemble_z(const double* __restrict__ Re, const double* __restrict__ Im, int nb,
                             cuDoubleComplex* __restrict__ Z) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)nb * nb;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % nb), j = (int)(t / nb);
    Z[t] = make_cuDoubleComplex(Re[(long long)i * nb + j], Im[(long long)i * nb + j]);
  }
}
// Z <- (Z + Z^H) / 2
__global__ void k_hermitian_part(cuDoubleComplex* Z, int n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % n), j = (int)(t / n);
    if (i < j) {
      const cuDoubleComplex a = Z[i + (long long)j * n], b = Z[j + (long long)i * n];
      const cuDoubleComplex m = make_cuDoubleComplex(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
      Z[i + (long long)j * n] = m;
      Z[j + (long long)i * n] = make_cuDoubleComplex(m.x, -m.y);
    } else if (i == j) {
      Z[t].y = 0.0;
    }
  }
}
__global__ void k_identity_z(cuDoubleComplex* I, int n) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x)
    I[t] = make_cuDoubleComplex((t % n) == (t / n) ? 1.0 : 0.0, 0.0);
}

// Complex S = dV X^H X (and, with HX, M = dV X^H (H X)) of FP32 interleaved bands, as FP64
// column-major complex matrices.  R4 holds four nb x nb real scratch matrices.
static int overlaps_cplx_mixed(Ctx& c, const float* X, const float* HX, int nb, double* R4, cuDoubleComplex* S,
                               cuDoubleComplex* M) {
  const size_t nn = (size_t)nb * nb;
  const int nparts = HX ? 4 : 2;
  RS_CUDA(cudaMemsetAsync(R4, 0, sizeof(double) * nn * nparts, c.stream));
  const float* parts[4] = {X, X, HX, HX};
  const int swap[4] = {0, 1, 0, 1};
  double* outs[4] = {R4, R4 + nn, R4 + 2 * nn, R4 + 3 * nn};
  const long long K = 2LL * (long long)c.ng;
  RS_TRY(gemm_tn_cat_x3(c, X, K, nb, parts, swap, nparts, K, nb, K, c.p.dv, outs, nb, c.gemm_terms_sm));
  k_assemble_z<<<64, 256, 0, c.stream>>>(outs[0], outs[1], nb, S);
  c.launches++;
  if (HX) {
    k_assemble_z<<<64, 256, 0, c.stream>>>(outs[2], outs[3], nb, M);
    c.launches++;
  }
  return check_launch("overlaps_cplx");
}

// zpotrf of S (upper) and T = R^-1 (upper triangle of S holds R afterwards)
static int cholesky_inverse_z(Ctx& c, int nb, cuDoubleComplex* S, cuDoubleComplex* T) {
  int lwork = 0, info = 0;
  RS_CUSOLVER(cusolverDnZpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, &lwork));
  RS_TRY(c.ws_solver.ensure(sizeof(cuDoubleComplex) * (size_t)std::max(lwork, 1)));
  RS_CUSOLVER(cusolverDnZpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<cuDoubleComplex>(), lwork,
                               c.ws_info.as<int>()));
  RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
  RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (zpotrf info=%d)", info);
  k_identity_z<<<64, 256, 0, c.stream>>>(T, nb);
  c.launches++;
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0);
  RS_CUBLAS(cublasZtrsm(c.cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nb, nb,
                        &one, S, nb, T, nb));
  return 0;
}

// gram_schmidt (Cholesky QR) and subspace_diag of complex FP32 bands; with both, the fused
// Cholesky-Rayleigh-Ritz step of the sweep (one rotation X <- X R^-1 V).
static int gssd_cplx_mixed(Ctx& c, int k, int s, bool gs, bool sd, double* h_esp) {
  const int nb = c.kp[k].nband;
  const size_t nn = (size_t)nb * nb;
  float* X = c.wfn(k, s).psi.as<float>();
  const long long ldx = 2LL * (long long)c.ng;
  RS_TRY(c.ws_dense.ensure(sizeof(cuDoubleComplex) * 4 * nn + sizeof(double) * (4 * nn + nb)));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  cuDoubleComplex* S = c.ws_dense.as<cuDoubleComplex>();
  cuDoubleComplex* M = S + nn;
  cuDoubleComplex* T = M + nn;
  cuDoubleComplex* U = T + nn;
  double* R4 = reinterpret_cast<double*>(U + nn);
  double* W = R4 + 4 * nn;
  float* HX = nullptr;
  if (sd) {
    RS_TRY(c.ws_hpsi.ensure(sizeof(float) * (size_t)ldx * nb));
    HX = c.ws_hpsi.as<float>();
    RS_TRY(hpsi_cplx<float>(c, k, s, X, HX, (size_t)ldx, nb));
  }
  RS_TRY(overlaps_cplx_mixed(c, X, HX, nb, R4, S, M));
  const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
  const cuDoubleComplex* C = nullptr;
  {
    ProfScope ps(c, "gs");
    if (gs) RS_TRY(cholesky_inverse_z(c, nb, S, T));
    if (sd) {
      k_hermitian_part<<<64, 256, 0, c.stream>>>(M, nb);
      c.launches++;
      if (gs) {  // Hsub = T^H M T of the orthonormalised block
        RS_CUBLAS(cublasZgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, M, nb, T, nb, &zero, U, nb));
        RS_CUBLAS(cublasZgemm(c.cublas, CUBLAS_OP_C, CUBLAS_OP_N, nb, nb, nb, &one, T, nb, U, nb, &zero, M, nb));
        k_hermitian_part<<<64, 256, 0, c.stream>>>(M, nb);
        c.launches++;
      }
    }
  }
  if (sd) {
    RS_TRY(eig_solve(c, nb, M, W));
    if (gs) {  // the single rotation R^-1 V
      RS_CUBLAS(cublasZgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, T, nb, M, nb, &zero, U, nb));
      C = U;
    } else {
      C = M;
    }
  } else {
    C = T;
  }
  RS_TRY(gemm_rotate_cx3(c, X, ldx, nb, (long long)c.ng, reinterpret_cast<const double*>(C), c.gemm_terms_rot));
  if (h_esp && sd) {
    RS_CUDA(cudaMemcpyAsync(h_esp, W, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return 0;
}

int gs_run(Ctx& c, int k, int s, int passes) {
  if (c.mixed && !c.cplx) return gs_mixed_real(c, k, s, passes);
  if (c.mixed && c.cplx) {
    for (int pass = 0; pass < std::max(1, passes); ++pass) RS_TRY(gssd_cplx_mixed(c, k, s, true, false, nullptr));
    return 0;
  }
  const int nb = c.kp[k].nband;
  const int ng = (int)c.ng;
  const size_t es = c.cplx ? sizeof(cuDoubleComplex) : sizeof(double);
  F64View v;
  RS_TRY(f64_view(c, k, s, v));
  RS_TRY(c.ws_dense.ensure(es * (size_t)nb * nb));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  int lwork = 0;
  if (c.cplx)
    RS_CUSOLVER(cusolverDnZpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, c.ws_dense.as<cuDoubleComplex>(),
                                            nb, &lwork));
  else
    RS_CUSOLVER(cusolverDnDpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, c.ws_dense.as<double>(), nb,
                                            &lwork));
  RS_TRY(c.ws_solver.ensure(es * (size_t)std::max(lwork, 1)));
  const double dV = c.p.dv, zero = 0.0, one = 1.0;
  const cuDoubleComplex zone = make_cuDoubleComplex(1.0, 0.0);
  ProfScope ps(c, "gs", 0.0, 2.0 * 2.0 * c.ng * (double)nb * nb * (c.cplx ? 4 : 1));
  for (int pass = 0; pass < std::max(1, passes); ++pass) {
    int info = 0;
    if (c.cplx) {
      cuDoubleComplex* S = c.ws_dense.as<cuDoubleComplex>();
      cuDoubleComplex* X = reinterpret_cast<cuDoubleComplex*>(v.x);
      RS_CUBLAS(cublasZherk(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, nb, ng, &dV, X, ng, &zero, S, nb));
      RS_CUSOLVER(cusolverDnZpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<cuDoubleComplex>(),
                                   lwork, c.ws_info.as<int>()));
      RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
      RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (zpotrf info=%d)", info);
      RS_CUBLAS(cublasZtrsm(c.cublas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, ng,
                            nb, &zone, S, nb, X, ng));
    } else {
      double* S = c.ws_dense.as<double>();
      if (nb <= kGramNbMax)
        RS_TRY(gram_small_f64(c, v.x, nullptr, ng, nb, dV, S, nullptr, false));
      else
        RS_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &dV, v.x, ng, &zero, S, nb));
      RS_CUSOLVER(cusolverDnDpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<double>(), lwork,
                                   c.ws_info.as<int>()));
      RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
      RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (potrf info=%d)", info);
      RS_CUBLAS(cublasDtrsm(c.cublas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, ng,
                            nb, &one, S, nb, v.x, ng));
    }
  }
  return f64_commit(c, k, s, v);
}

int sd_run(Ctx& c, int k, int s, double* h_esp) {
  if (c.mixed && !c.cplx) return sd_mixed_real(c, k, s, h_esp);
  if (c.mixed && c.cplx) return gssd_cplx_mixed(c, k, s, false, true, h_esp);
  const int nb = c.kp[k].nband;
  const int ng = (int)c.ng;
  const size_t es = c.cplx ? sizeof(cuDoubleComplex) : sizeof(double);
  F64View v;
  RS_TRY(f64_view(c, k, s, v));
  RS_TRY(c.ws_hpsi.ensure(sizeof(double) * nreal(c) * nb));
  double* HX = c.ws_hpsi.as<double>();
  if (c.cplx)
    RS_TRY(hpsi_cplx<double>(c, k, s, v.x, HX, nreal(c), nb));
  else
    RS_TRY(hpsi_real<double>(c, k, s, v.x, HX, c.ng, nb));
  RS_TRY(c.ws_dense.ensure(es * (size_t)nb * nb + sizeof(double) * nb));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* W = reinterpret_cast<double*>(c.ws_dense.as<char>() + es * (size_t)nb * nb);
  const double hdV = 0.5 * c.p.dv, zero = 0.0, one = 1.0;
  const cuDoubleComplex zhdV = make_cuDoubleComplex(hdV, 0.0), zone = make_cuDoubleComplex(1.0, 0.0),
                        zzero = make_cuDoubleComplex(0.0, 0.0);
  {
    ProfScope ps(c, "sd_gemm", 0.0, 2.0 * c.ng * (double)nb * nb * (c.cplx ? 4 : 1));
    if (c.cplx)
      RS_CUBLAS(cublasZher2k(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_C, nb, ng, &zhdV,
                             reinterpret_cast<cuDoubleComplex*>(v.x), ng, reinterpret_cast<cuDoubleComplex*>(HX), ng,
                             &zero, c.ws_dense.as<cuDoubleComplex>(), nb));
    else if (nb <= kGramNbMax)
      RS_TRY(gram_small_f64(c, v.x, HX, ng, nb, c.p.dv, nullptr, c.ws_dense.as<double>(), true));
    else
      RS_CUBLAS(cublasDsyr2k(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &hdV, v.x, ng, HX, ng, &zero,
                             c.ws_dense.as<double>(), nb));
  }
  RS_TRY(eig_solve(c, nb, c.ws_dense.p, W));
  ProfScope ps(c, "sd_rot", 0.0, 2.0 * c.ng * (double)nb * nb * (c.cplx ? 4 : 1));
  // rotation Psi <- Psi V in grid chunks (out of place per chunk, then copied back)
  size_t ch = std::max<size_t>(1024, (size_t)(256u << 20) / (es * (size_t)nb));
  ch = std::min<size_t>(ch, c.ng);
  RS_TRY(c.ws_rot.ensure(es * ch * nb));
  for (size_t g0 = 0; g0 < c.ng; g0 += ch) {
    const int m = (int)std::min(ch, c.ng - g0);
    if (c.cplx) {
      cuDoubleComplex* X = reinterpret_cast<cuDoubleComplex*>(v.x);
      RS_CUBLAS(cublasZgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &zone, X + g0, ng,
                            c.ws_dense.as<cuDoubleComplex>(), nb, &zzero, c.ws_rot.as<cuDoubleComplex>(), m));
      RS_CUDA(cudaMemcpy2DAsync(X + g0, es * c.ng, c.ws_rot.p, es * m, es * m, nb, cudaMemcpyDeviceToDevice, c.stream));
    } else {
      RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &one, v.x + g0, ng, c.ws_dense.as<double>(),
                            nb, &zero, c.ws_rot.as<double>(), m));
      RS_CUDA(cudaMemcpy2DAsync(v.x + g0, es * c.ng, c.ws_rot.p, es * m, es * m, nb, cudaMemcpyDeviceToDevice, c.stream));
    }
  }
  if (h_esp) {
    RS_CUDA(cudaMemcpyAsync(h_esp, W, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return f64_commit(c, k, s, v);
}

// One Gram-Schmidt + subspace_diag step of the sweep (real build) as a Cholesky-Rayleigh-Ritz
// with a single rotation: S = dV X^T X, M = dV X^T (H X), S = R^T R, Hsub = R^-T M R^-1 =
// V diag(e) V^T, X <- X (R^-1 V).  In exact arithmetic this is gram_schmidt (the Q factor of
// X = Q R, src/gram_schmidt/gram_schmidt_t_module.f90:85-308) followed by subspace_diag_la
// (src/subspace_diag/subspace_diag_la_module.f90:18-223): H is linear, so H (X R^-1) =
// (H X) R^-1 and Hsub of the orthonormalised block is R^-T M R^-1; the orthonormalised block is
// never formed, which saves one of the four ng x nb x nb contractions per sweep.
int gssd_run(Ctx& c, int k, int s, double* h_esp, bool use_cg_hx) {
  if (c.cplx && c.mixed) return gssd_cplx_mixed(c, k, s, true, true, h_esp);
  if (c.cplx) {
    RS_TRY(gs_run(c, k, s, 1));
    return sd_run(c, k, s, h_esp);
  }
  const int nb = c.kp[k].nband;
  const int ng = (int)c.ng;
  RS_TRY(c.ws_dense.ensure(sizeof(double) * (3 * (size_t)nb * nb + nb)));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* S = c.ws_dense.as<double>();
  double* M = S + (size_t)nb * nb;
  double* T = M + (size_t)nb * nb;
  double* W = T + (size_t)nb * nb;
  const double dV = c.p.dv, zero = 0.0, one = 1.0;
  F64View v;
  float* X32 = nullptr;
  // H X of the bands as CG left them (kept up to date by its line-search updates), when the
  // CG that just ran covered every band of (k, s) in one array and rejected no step
  bool reuse = use_cg_hx && c.cg_hx_ready && c.cg_hx_k == k && c.cg_hx_s == s &&
               c.ws_hpsi.bytes >= (c.mixed ? sizeof(float) : sizeof(double)) * c.ng * nb;
  c.cg_hx_ready = false;
  if (reuse) {
    int rejected = 0;
    RS_CUDA(cudaMemcpyAsync(&rejected, c.ws_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    reuse = rejected == 0;
  }
  if (c.mixed) {
    X32 = c.wfn(k, s).psi.as<float>();
    RS_TRY(c.ws_hpsi.ensure(sizeof(float) * c.ng * nb));
    float* HX = c.ws_hpsi.as<float>();
    if (!reuse) RS_TRY(hpsi_real<float>(c, k, s, X32, HX, c.ng, nb));
    RS_CUDA(cudaMemsetAsync(S, 0, sizeof(double) * 2 * (size_t)nb * nb, c.stream));
    RS_TRY(gemm_tn2_x3(c, X32, HX, (long long)c.ng, nb, (long long)c.ng, dV, S, M, c.gemm_terms_sm));
  } else {
    RS_TRY(f64_view(c, k, s, v));
    RS_TRY(c.ws_hpsi.ensure(sizeof(double) * c.ng * nb));
    double* HX = c.ws_hpsi.as<double>();
    if (!reuse) RS_TRY(hpsi_real<double>(c, k, s, v.x, HX, c.ng, nb));
    ProfScope ps(c, "sd_gemm", 0.0, 2.0 * 2.0 * c.ng * (double)nb * nb);
    // S and M = dV X^T (H X) are symmetric (H is): their upper triangles only
    if (nb <= kGramNbMax) {
      RS_TRY(gram_small_f64(c, v.x, HX, ng, nb, dV, S, M, false));
    } else {
      RS_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &dV, v.x, ng, &zero, S, nb));
      RS_CUBLAS(cublasDsyrkx(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &dV, v.x, ng, HX, ng, &zero, M,
                             nb));
    }
  }
  {
    ProfScope ps(c, "gs");
    if (!c.mixed || c.gemm_tri == 2)
      k_fill_lower<<<64, 256, 0, c.stream>>>(M, nb);  // the upper triangle of M was formed
    else
      k_symmetrize<<<64, 256, 0, c.stream>>>(M, nb);  // both triangles were formed: average
    c.launches++;
    int lwork = 0;
    RS_CUSOLVER(cusolverDnDpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, &lwork));
    RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
    RS_CUSOLVER(cusolverDnDpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<double>(), lwork,
                                 c.ws_info.as<int>()));
    int info = 0;
    RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
    RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (potrf info=%d)", info);
    // T <- R^-1 (upper triangle of S holds R)
    k_identity<<<64, 256, 0, c.stream>>>(T, nb);
    c.launches++;
    RS_CUBLAS(cublasDtrsm(c.cublas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, nb, nb,
                          &one, S, nb, T, nb));
    // S <- M R^-1 ; M <- R^-T (M R^-1) = Hsub
    RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, M, nb, T, nb, &zero, S, nb));
    RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_T, CUBLAS_OP_N, nb, nb, nb, &one, T, nb, S, nb, &zero, M, nb));
    k_symmetrize<<<64, 256, 0, c.stream>>>(M, nb);
    c.launches++;
  }
  RS_TRY(eig_solve(c, nb, M, W));
  // S <- R^-1 V: the single rotation
  RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, nb, nb, nb, &one, T, nb, M, nb, &zero, S, nb));
  if (c.mixed) {
    if (c.rot_update) {
      k_rotation_update_form<<<nb, 256, 0, c.stream>>>(S, nb);
      c.launches++;
    }
    RS_TRY(gemm_rotate_x3(c, X32, (long long)c.ng, nb, (long long)c.ng, S, nb, c.gemm_terms_rot, c.rot_update != 0));
  } else {
    ProfScope ps(c, "sd_rot", 0.0, 2.0 * c.ng * (double)nb * nb);
    size_t ch = std::max<size_t>(1024, (size_t)(256u << 20) / (sizeof(double) * (size_t)nb));
    ch = std::min<size_t>(ch, c.ng);
    RS_TRY(c.ws_rot.ensure(sizeof(double) * ch * nb));
    for (size_t g0 = 0; g0 < c.ng; g0 += ch) {
      const int m = (int)std::min(ch, c.ng - g0);
      RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &one, v.x + g0, ng, S, nb, &zero,
                            c.ws_rot.as<double>(), m));
      RS_CUDA(cudaMemcpy2DAsync(v.x + g0, sizeof(double) * c.ng, c.ws_rot.p, sizeof(double) * m,
                                sizeof(double) * m, nb, cudaMemcpyDeviceToDevice, c.stream));
    }
  }
  if (h_esp) {
    RS_CUDA(cudaMemcpyAsync(h_esp, W, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return c.mixed ? 0 : f64_commit(c, k, s, v);
}

}  // namespace rsdft
