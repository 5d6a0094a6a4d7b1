// Dense band-space operations: Gram-Schmidt (Cholesky QR) and subspace diagonalisation.
//
// Reference semantics:
//   gram_schmidt_t (src/gram_schmidt/gram_schmidt_t_module.f90:85-308) orthonormalises the
//   bands in order with the dV inner product; its result is the Q factor of Psi = Q R with
//   R upper triangular and positive diagonal.  Cholesky QR (the reference's GS=4 variant,
//   src/gram_schmidt/gram_schmidt_lusl_module.f90:241-328: S = dV Psi^T Psi, potrf, trtri,
//   Psi <- Psi R^-1) produces the same Q, with O(N M^2) GEMM work instead of a recursion.
//   subspace_diag_la (src/subspace_diag/subspace_diag_la_module.f90:18-223):
//   Hsub = 1/2 dV (Psi^T H Psi + (H Psi)^T Psi) (dsyr2k), dsyev, Psi <- Psi V.
// FP64 path: cuBLAS dsyrk/dsyr2k/dtrsm/dgemm and cuSOLVER dpotrf/dsyevd.
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

static int f64_view(Ctx& c, int k, int s, F64View& v, DBuf& tmp) {
  const int nb = c.kp[k].nband;
  if (!c.mixed) {
    v.x = c.wfn(k, s).psi.as<double>();
    return 0;
  }
  RS_TRY(tmp.ensure(sizeof(double) * c.ng * nb));
  RS_TRY(convert_f2d(c, c.wfn(k, s).psi.as<float>(), tmp.as<double>(), c.ng * nb));
  v.x = tmp.as<double>();
  v.converted = true;
  return 0;
}
static int f64_commit(Ctx& c, int k, int s, F64View& v) {
  if (!v.converted) return 0;
  return convert_d2f(c, v.x, c.wfn(k, s).psi.as<float>(), c.ng * c.kp[k].nband);
}



static int read_info(Ctx& c, int* d_info, int* h_info) {
  RS_CUDA(cudaMemcpyAsync(h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return 0;
}

int gs_run(Ctx& c, int k, int s, int passes) {
  RS_CHECK(!c.cplx, RSDFT_ERR_UNSUPPORTED, "complex16 GS is provided by gs_cplx");
  const int nb = c.kp[k].nband;
  const int ng = (int)c.ng;
  F64View v;
  RS_TRY(f64_view(c, k, s, v, c.ws_f64));
  RS_TRY(c.ws_dense.ensure(sizeof(double) * (size_t)nb * nb));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* S = c.ws_dense.as<double>();
  int lwork = 0;
  RS_CUSOLVER(cusolverDnDpotrf_bufferSize(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, &lwork));
  RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
  const double dV = c.p.dv, zero = 0.0, one = 1.0;
  ProfScope ps(c, "gs");
  for (int pass = 0; pass < std::max(1, passes); ++pass) {
    RS_CUBLAS(cublasDsyrk(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &dV, v.x, ng, &zero, S, nb));
    RS_CUSOLVER(cusolverDnDpotrf(c.cusolver, CUBLAS_FILL_MODE_UPPER, nb, S, nb, c.ws_solver.as<double>(), lwork,
                                 c.ws_info.as<int>()));
    int info = 0;
    RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
    RS_CHECK(info == 0, RSDFT_ERR_NOT_SPD, "overlap matrix not positive definite (potrf info=%d)", info);
    RS_CUBLAS(cublasDtrsm(c.cublas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, ng,
                          nb, &one, S, nb, v.x, ng));
    c.launches += 3;
  }
  return f64_commit(c, k, s, v);
}

int sd_run(Ctx& c, int k, int s, double* h_esp) {
  RS_CHECK(!c.cplx, RSDFT_ERR_UNSUPPORTED, "complex16 SD is provided by sd_cplx");
  const int nb = c.kp[k].nband;
  const int ng = (int)c.ng;
  F64View v;
  RS_TRY(f64_view(c, k, s, v, c.ws_f64));
  RS_TRY(c.ws_hpsi.ensure(sizeof(double) * c.ng * nb));
  double* HX = c.ws_hpsi.as<double>();
  RS_TRY(hpsi_real<double>(c, k, s, v.x, HX, c.ng, nb));
  RS_TRY(c.ws_dense.ensure(sizeof(double) * ((size_t)nb * nb + nb)));
  RS_TRY(c.ws_info.ensure(sizeof(int) * 4));
  double* H = c.ws_dense.as<double>();
  double* W = H + (size_t)nb * nb;
  const double hdV = 0.5 * c.p.dv, zero = 0.0, one = 1.0;
  ProfScope ps(c, "sd");
  RS_CUBLAS(cublasDsyr2k(c.cublas, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_T, nb, ng, &hdV, v.x, ng, HX, ng, &zero, H, nb));
  int lwork = 0;
  RS_CUSOLVER(cusolverDnDsyevd_bufferSize(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, H, nb, W,
                                          &lwork));
  RS_TRY(c.ws_solver.ensure(sizeof(double) * (size_t)std::max(lwork, 1)));
  RS_CUSOLVER(cusolverDnDsyevd(c.cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, nb, H, nb, W,
                               c.ws_solver.as<double>(), lwork, c.ws_info.as<int>()));
  int info = 0;
  RS_TRY(read_info(c, c.ws_info.as<int>(), &info));
  RS_CHECK(info == 0, RSDFT_ERR_EIG, "subspace eigensolver failed (syevd info=%d)", info);
  // rotation Psi <- Psi V in grid chunks (out of place per chunk, then copied back)
  size_t ch = std::max<size_t>(1024, (size_t)(256u << 20) / (sizeof(double) * (size_t)nb));
  ch = std::min<size_t>(ch, c.ng);
  RS_TRY(c.ws_rot.ensure(sizeof(double) * ch * nb));
  double* tmp = c.ws_rot.as<double>();
  for (size_t g0 = 0; g0 < c.ng; g0 += ch) {
    const int m = (int)std::min(ch, c.ng - g0);
    RS_CUBLAS(cublasDgemm(c.cublas, CUBLAS_OP_N, CUBLAS_OP_N, m, nb, nb, &one, v.x + g0, ng, H, nb, &zero, tmp, m));
    RS_CUDA(cudaMemcpy2DAsync(v.x + g0, sizeof(double) * c.ng, tmp, sizeof(double) * m, sizeof(double) * m, nb,
                              cudaMemcpyDeviceToDevice, c.stream));
    c.launches += 2;
  }
  c.launches += 3;
  if (h_esp) {
    RS_CUDA(cudaMemcpyAsync(h_esp, W, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return f64_commit(c, k, s, v);
}

}  // namespace rsdft
