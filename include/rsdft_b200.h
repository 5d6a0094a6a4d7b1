/*
 * rsdft_b200.h -- C ABI of the B200 (sm_100a) band-update library for RSDFT.
 *
 * The library replaces the four module procedures of RSDFT_DEVELOP's band
 * update with CUDA implementations that keep the wavefunctions resident in HBM:
 *
 *   hamiltonian(tpsi, htpsi, n, k, s)            src/hamiltonian_module.f90:44-46,118-172
 *   conjugate_gradient(n1, n2, k, s, unk, esp, res)
 *                                                src/conjugate_gradient/cg_module.f90:53-109
 *   gram_schmidt(n0, n1, k, s)                   src/gram_schmidt/gram_schmidt_module.f90:35-79
 *   subspace_diag(k, s, unk, esp)                src/subspace_diag/subspace_diag_module.f90:17-32
 *
 * plus the sweep driver order of calc_sweep (src/sweep_module.f90:148-215).
 *
 * Conventions (chosen so a Fortran ISO_C_BINDING shim can pass its arrays as is):
 *  - k, s, band and grid indices are 1-based, as in the reference;
 *  - wavefunction blocks are Fortran column-major unk(ML0, nb): band-major,
 *    grid index j = 1 + i1 + i2*N1 + i3*N1*N2 (x fastest,
 *    src/kinetic/d_kinetic_sol_module.f90:129);
 *  - complex16 arrays are interleaved (re, im) pairs, i.e. Fortran complex(8);
 *  - every entry returns RSDFT_OK (0) or a negative status; it never aborts.
 *    rsdft_gpu_last_error() gives the message of the last failure (the
 *    reference instead calls stop_program, e.g. src/hamiltonian_module.f90:396).
 *  - single-threaded host use: one implicit context per process, one CUDA
 *    stream; not re-entrant (the reference calls these from the serial part of
 *    its OpenMP code, src/hamiltonian_module.f90:123-140).
 */
#ifndef RSDFT_B200_H
#define RSDFT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define RSDFT_OK               0
#define RSDFT_ERR_ARG         -1   /* invalid argument / size */
#define RSDFT_ERR_OOM         -2   /* device allocation failed */
#define RSDFT_ERR_CUDA        -3   /* CUDA runtime / library error */
#define RSDFT_ERR_NOT_SPD     -4   /* overlap matrix not positive definite (Cholesky) */
#define RSDFT_ERR_EIG         -5   /* dense eigensolver failed */
#define RSDFT_ERR_TIMEOUT     -6   /* a bounded device-side wait gave up */
#define RSDFT_ERR_STATE       -7   /* call order (init/set_* missing) */
#define RSDFT_ERR_UNSUPPORTED -8   /* configuration not built in */
#define RSDFT_ERR_NUMERIC     -9   /* NaN/Inf detected in inputs or results */
#define RSDFT_ERR_IO          -10  /* file open / read / write error or malformed file */

/* ---- precision modes ---- */
#define RSDFT_PREC_FP64   0  /* all FP64 (the plain GPU drop-in) */
#define RSDFT_PREC_MIXED  1  /* FP32 stencils/CG, split-BF16 GEMMs, FP64 dense solves + residuals */

/* ---- preconditioner modes (SWPC in the reference, src/conjugate_gradient/cg_module.f90:27) ---- */
#define RSDFT_PC_NONE      0
#define RSDFT_PC_HPRSDFT   4   /* precond_hprsdft: mloop CG steps on the 7-point -1/2 Laplacian */
#define RSDFT_PC_LEARNED 100   /* learned 3-D conv preconditioner, hprsdft fallback */

/* ---- memory spaces for pointer arguments ---- */
#define RSDFT_MEM_HOST    0
#define RSDFT_MEM_DEVICE  1

#define RSDFT_MDMAX 12

/* Operator/grid description; mirrors init_kinetic + rgrid_module state
 * (src/kinetic/kinetic_module.f90:28-162, src/rgrid_sol_module.f90:25-38). */
typedef struct rsdft_gpu_params {
  int n1, n2, n3;                 /* Ngrid(1:3) */
  int md;                         /* FD half order Md (4 or 6 built in) */
  double hgrid[3];                /* Hgrid(1:3) */
  double dv;                      /* dV */
  double coef_lap[3][RSDFT_MDMAX];/* coef_lap(d, m), m = 1..Md */
  double coef_lap0;               /* coef_lap0 */
  double ggg[3];                  /* ggg(1:3); preconditioner c0 = sum ggg/H^2 */
  int nk;                         /* k-points held by this context */
  int nspin;                      /* spins held by this context */
  int mb;                         /* bands per (k, s) (maximum) */
  int is_complex;                 /* 0: real8/Gamma build, 1: complex16 build */
  int precision;                  /* RSDFT_PREC_* */
  int pc_mode;                    /* RSDFT_PC_* */
  int ncg;                        /* Ncg (default 3) */
  int mloop;                      /* preconditioner inner steps (default 3) */
  int cg_block;                   /* MB_d bands per batched CG block (0: automatic) */
} rsdft_gpu_params;

/* ---- context ---- */
int rsdft_gpu_init(const rsdft_gpu_params* p);
int rsdft_gpu_finalize(void);
const char* rsdft_gpu_last_error(void);
int rsdft_gpu_get_stream(void** stream);              /* the library's cudaStream_t */
int rsdft_gpu_synchronize(void);

/* ---- operator set-up ---- */
/* k-dependent kinetic terms (coef_nabk(3,Md,k), const_k2(k); kinetic_module.f90:141-162)
 * and the active band count of this k-point. */
int rsdft_gpu_set_kpoint(int k, const double coef_nabk[3][RSDFT_MDMAX], double const_k2, int nband);
/* Vloc(ML0, s) (src/localpot_module.f90:40-87). */
int rsdft_gpu_set_vloc(const double* vloc, int ml, int s);
/* Projector tables in the reference layout: MJJ(nzlma), JJP(MAXMJJ,nzlma) (1-based grid
 * indices), amap(nzlma) atom of each projector, and the coupling in nzqr_pair(2,npair) /
 * Dij00(npair) form (src/ps_nloc_mr_module.f90:852-897).  The KB form of
 * src/d_ps_nloc2_op_module.f90 is npair = nzlma with pairs (p,p) and Dij00 = iuV(p).
 * Pairs must couple projectors of the same atom. */
int rsdft_gpu_set_projectors(int nzlma, int maxmjj, const int* mjj, const int* jjp,
                             const int* amap, int npair, const int* pairs, const double* dij00);
/* d_uVk(MAXMJJ, nzlma, k) / z_uVk(MAXMJJ, nzlma, k) for one k (ps_nloc2_module.f90:1070-1167). */
int rsdft_gpu_set_uvk_d(int k, const double* uvk);
int rsdft_gpu_set_uvk_z(int k, const double* uvk_interleaved);

/* ---- wavefunctions (resident on the device between calls) ---- */
int rsdft_gpu_set_wf_d(int k, int s, const double* unk, int ld, int nb);
int rsdft_gpu_get_wf_d(int k, int s, double* unk, int ld, int nb);
int rsdft_gpu_set_wf_z(int k, int s, const double* unk, int ld, int nb);
int rsdft_gpu_get_wf_z(int k, int s, double* unk, int ld, int nb);
/* Seeded device-side initial wavefunctions (replaces random_initial_wf,
 * src/wf_module.f90:161-191): element e = ((k0*2^20 + band0)*ML0 + j)*2 + reim holds
 * sum_{t<12} u(e,t) - 6, u = (splitmix64(seed*2^40 + 12e + t) >> 11) * 2^-53. */
int rsdft_gpu_random_wf(int k, int s, uint64_t seed);
/* Wavefunction restart files in the reference's format: write_wf_simple
 * (src/io_write_wf_simple_module.f90:21-276, IO_ctrl = 0, OC < 10) via write_data
 * (src/io_module.f90:59-259).  Writes bands 1..MB of every (k, s) of the resident unk as a Fortran
 * sequential unformatted file (4-byte record markers): header (-1, ML.., MB.., MK MS MMBZ,
 * IO_ctrl OC TYPE_WF), LL2 grid map, occ(MB,MK,MS), aa, bb, kbb(3,MK), one-process parallel
 * info, then one record per band (s, k, n order) in FP64 (oc 1, 3) or FP32 (oc 4, 5).  occ, aa,
 * bb, kbb are host arrays of the caller (NULL writes zeros); MB is the largest band count over
 * the k-points, bands past a k-point's own count are written as zeros. */
int rsdft_gpu_write_wf(const char* path, int oc, const double* occ, const double* aa, const double* bb,
                       const double* kbb);
/* read_wf_simple (src/io_read_wf_simple_module.f90:21-560, IO_ctrl = 0): reads a file of either
 * layout (new, or the old one without the leading -1), FP64 or FP32, real or complex records,
 * into the resident unk of every (k, s), placing each point by the file's LL2 grid map.  The grid
 * and the k-point / spin counts must match the context; occ (MB x MK x MS, may be NULL) receives
 * the file's occupations.  A complex file read by a real context keeps the real part; a real file
 * read by a complex context gets zero imaginary parts (as the reference does). */
int rsdft_gpu_read_wf(const char* path, double* occ);

/* ---- the four module procedures ---- */
/* hamiltonian: htpsi(:,1:nb) = H tpsi(:,1:nb) (overwrites htpsi).  mem selects host or device
 * pointers; _f is the FP32 variant on FP32 arrays. */
int rsdft_gpu_hamiltonian_d(int k, int s, const double* tpsi, double* htpsi, int ld, int nb, int mem);
int rsdft_gpu_hamiltonian_z(int k, int s, const double* tpsi, double* htpsi, int ld, int nb, int mem);
int rsdft_gpu_hamiltonian_f(int k, int s, const float* tpsi, float* htpsi, int ld, int nb, int mem);
int rsdft_gpu_hamiltonian_c(int k, int s, const float* tpsi, float* htpsi, int ld, int nb, int mem);
/* hamiltonian on caller-owned DEVICE blocks (FP64, real8 build) that performs no device
 * allocation.  No counterpart in the reference.  For callers that cannot let a library call
 * cudaMalloc -- a host code that reserves the whole device memory pool up front, a caller
 * running inside another framework's memory pool, or a loop where cudaMalloc's implicit device
 * synchronisation would stall -- the nonlocal coefficient scratch comes from a fixed 4 MiB array
 * compiled into the library (held on every GPU that loads it until the process exits):
 * nb x (atoms x padded projectors per atom) must not exceed 524288, larger requests return
 * RSDFT_ERR_ARG (split the bands into blocks).  The first call of a context looks the array's
 * device address up (cudaGetSymbolAddress, on the device that was current at rsdft_gpu_init;
 * another current device returns RSDFT_ERR_STATE); make that first call before any stream
 * capture.  The stencil runs in its stencil + scatter form whatever rsdft_gpu_set_nl_form
 * selects (no tuning runs, no host synchronisation).  All calls share the array: calls that
 * overlap on the GPU race; nothing in it has to start at zero (every call rewrites what it
 * reads).  Runs on the library stream. */
int rsdft_gpu_hamiltonian_noalloc_d(int k, int s, const double* tpsi, double* htpsi, int ld, int nb);
/* conjugate_gradient on the resident unk(:,:,k,s); esp/res (host, length nband) as the
 * reference's esp(:,k,s)/res(:,k,s), res = dV |H psi - e psi|^2 (cg_module.f90:231,556). */
int rsdft_gpu_conjugate_gradient(int k, int s, double* esp, double* res);
/* gram_schmidt(1, nband, k, s) on the resident unk (Cholesky-QR on the device). */
int rsdft_gpu_gram_schmidt(int k, int s);
/* subspace_diag(k, s, unk, esp): Rayleigh-Ritz on the resident unk; esp may be NULL. */
int rsdft_gpu_subspace_diag(int k, int s, double* esp);
/* FP64 residual check of the resident unk: esp = <x|Hx>/<x|x>, res = dV|Hx-esp x|^2/<x|x>dV. */
int rsdft_gpu_residual(int k, int s, double* esp, double* res);
/* Preconditioner alone (precond_hprsdft): pgk = P gk; test entry. */
int rsdft_gpu_precond_d(int k, const double* gk, double* pgk, int ld, int nb, int mem);
/* The same on FP32 bands, as mixed-precision CG runs it: the mloop CG steps evaluated in the
 * s-step (Krylov-basis) form, 3 mloop + 3 passes over the bands (mloop <= 4). */
int rsdft_gpu_precond_f(int k, const float* gk, float* pgk, int ld, int nb, int mem);
/* FP32 precond_hprsdft form inside conjugate_gradient: 3 (default) the s-step form in 3 mloop + 3
 * passes, the last one forming the CG direction p = Pg + beta p itself (<Pg|g> from the Krylov
 * moments, src/conjugate_gradient/cg_module.f90:254-283; with SWGS on it runs as form 1),
 * 1 the same passes leaving Pg for separate <Pg|g> and direction passes,
 * 2 the s-step form fused into two z-streamed passes together with <Pg|g> and the direction
 * update (mloop 1..3, SWGS off), 0 the recurrence form of the FP64 path.
 * rsdft_gpu_precond_f uses form 1 for 1, 2 and 3. */
int rsdft_gpu_set_pc_form(int form);
/* Orthogonalisation of the preconditioned gradient inside conjugate_gradient, the reference's
 * SWGS keyword (src/conjugate_gradient/cg_module.f90:47, cggs at :249-251 and :576-578):
 * 0 off (the default), 1 cggs_1 (against the bands below, src/conjugate_gradient/
 * cggs_module.f90:36-76), 2 cggs_2 (against all other bands, :79-121).  Bands of earlier CG
 * blocks (cg_block) count with their updated values, bands of the same block with their values
 * at the same CG step, as with the reference's MB_d blocks. */
int rsdft_gpu_set_cggs(int iswitch);

/* calc_sweep: up to nsweep iterations of CG -> GS -> SD over all (k, s); stops early when the
 * FP64 residual max over bands <= tol (tol <= 0: never).  The FP64 residual is evaluated in
 * the sweeps where CG's own residual of the bands it returned is within 30 x tol (and in the
 * last).  iters receives the sweeps done; esp/res (host, nband*nk*nspin, k-major after band)
 * receive the final FP64 values. */
int rsdft_gpu_sweep(int nsweep, double tol, int* iters, double* esp, double* res);
/* Switch the context between RSDFT_PREC_MIXED and RSDFT_PREC_FP64, converting the resident
 * wavefunctions of every (k, s) (to FP32 by rounding, to FP64 exactly).  The FP64 final polish of
 * a mixed-precision solve: rsdft_gpu_sweep to the FP32 floor (res ~ 1e-9 .. 1e-10) in mixed
 * precision, then rsdft_gpu_set_precision(RSDFT_PREC_FP64) and rsdft_gpu_sweep to the tighter
 * tolerance.  No counterpart in the reference (which has one precision per build). */
int rsdft_gpu_set_precision(int precision);
/* Convergence band set of rsdft_gpu_sweep: bands 1..mb_ref are checked (0: all bands), as the
 * reference's init_sweep(iconv_check, mb_ref, tol) does for its band and DOS drivers
 * (src/sweep_module.f90:46-60,267-278; src/band_module.f90:207; src/dos_module.f90:64-75).
 * mb_ref = -1: per k-point, bands 1..nband_k - nband_k/8 (k-points with uneven band counts). */
int rsdft_gpu_init_sweep(int mb_ref);
/* Convergence test of rsdft_gpu_sweep: 0 (default) max over bands 1..mb_ref of the FP64 residual
 * res(n) <= tol; 2 the reference's conv_check_2 (src/sweep_module.f90:277-288), used by its band
 * driver (init_sweep(2, mb2_band, esp_conv_tol), src/band_module.f90:207): no eigenvalue of bands
 * 1..mb_ref moved by tol or more in the last sweep.  esp/res returned are the FP64 residual
 * check's values of the last sweep. */
int rsdft_gpu_set_sweep_check(int iconv_check);

/* ---- SCF pieces (the caller of the band update, src/scf_module.f90:85-563) ----
 * V_ion: the fixed local potential (localpot_module Vion); Vloc(:,s) = Vion + Vh + Vxc(:,s)
 * (src/localpot_module.f90:209-215) once rsdft_gpu_potential has run. */
int rsdft_gpu_set_vion(const double* vion, int ml);
/* The device density rho(ML, nspin) from the host (initial density, restart) / back to the
 * host with the Hartree and XC potentials of the last rsdft_gpu_potential (any may be NULL). */
int rsdft_gpu_set_rho(const double* rho, int ml);
int rsdft_gpu_get_rho(double* rho, double* vh, double* vxc);
/* calc_density (src/density_module.f90): rho(:,s) = sum_{k,n} occ(n,k,s) |unk(:,n,k,s)|^2 from
 * the resident bands; occ (MB, MK, MS) host, Fortran order, k-point weights and spin factor
 * included as calc_fermi leaves them. */
int rsdft_gpu_density(const double* occ);
/* normalize_density: scale rho to nelec electrons. */
int rsdft_gpu_normalize_density(double nelec);
/* calc_hartree (FFT Poisson: V_H(G) = 4 pi rho(G)/|G|^2, G != 0) + calc_xc (LDA PZ81,
 * src/xc/xc_ldapz81_module.f90) from the device density, then Vloc(:,s) = Vion + Vh + Vxc(:,s)
 * on the device.  ene (4, may be NULL): E_H = 1/2 int rho V_H, E_xc, int rho V_xc, charge. */
int rsdft_gpu_potential(double* ene);
/* init_mixing (src/mixing/mixing_module.f90:70-142) for IMIX = 10 (Pulay on the density) with
 * history mmix (1..8) and beta: Xold = (rho, Vloc) of now. */
int rsdft_gpu_init_mixing(int mmix, double beta);
/* calc_sqerr (src/mixing/mixing_module.f90:319-341): sqerr(1:MS) of Vloc, sqerr(MS+1:2MS) of rho
 * against Xold, each sum of squares / ML. */
int rsdft_gpu_sqerr(double* sqerr);
/* perform_mixing (src/mixing/mixing_module.f90:145-298) with pulay_mixing
 * (src/mixing/mixing_pulay_module.f90:29-111): the device density becomes the mixed one
 * (beta search for beta > 1 as the reference); beta_used (may be NULL) receives the beta taken. */
int rsdft_gpu_mix_density(double* beta_used);
/* GGA-PBE exchange-correlation potential of the host density rho (nspin x ML0, Fortran order
 * rho(ML0, nspin)), as calc_GGAPBE96_2 forms it (src/xc/xc_ggapbe96_2_module.f90:26-370: FD
 * gradient of the total density of order Md, densities <= 1e-10 skipped): vxc (nspin x ML0,
 * host) and, if exc is not NULL, exc[0] = E_x, exc[1] = E_c.  Uses the context's grid, H and
 * Md (<= 6); the gradient is taken along the grid axes with 1/H per axis (orthorhombic cells). */
int rsdft_gpu_xc_pbe(const double* rho, double* vxc, double* exc);

/* ---- learned preconditioner (no counterpart in the reference) ----
 * A 4-layer 3-D convolutional network, channels 1-16-16-16-1, 3x3x3 kernels, no biases, tanh
 * between layers, BF16 weights with FP32 accumulation.  With pc_mode RSDFT_PC_LEARNED and
 * RSDFT_PREC_MIXED it replaces precond_hprsdft (src/conjugate_gradient/cgpc_hprsdft_module.f90:
 * 133-270) in conjugate_gradient: Pg = rms(g) f(g / rms(g)) per band.  Until weights are
 * loaded or trained, and in other builds, precond_hprsdft runs instead; rsdft_gpu_sweep also
 * falls back to it for good when the FP64 residual stalls for 3 sweeps.
 * Weights are RSDFT_LPC_NWEIGHTS FP32 values, layer by layer, each [cout][cin][kz][ky][kx]. */
#define RSDFT_LPC_NWEIGHTS 14688
/* Random initial weights (normal, variance 1/(27 cin)). */
int rsdft_gpu_lpc_init(unsigned long long seed);
int rsdft_gpu_lpc_set_weights(const float* w, int n);
int rsdft_gpu_lpc_get_weights(float* w, int n);
/* Network output y = f(x) for nb fields of n1 x n2 x n3 (x fastest); periodic (1) or zero (0)
 * padding; no input scaling. */
int rsdft_gpu_lpc_forward(const float* x, float* y, int nb, int n1, int n2, int n3, int periodic,
                          int mem);
/* Mean squared error over the interior (margin points in from every face) of nb zero-padded
 * n^3 patches, and its gradient with respect to the FP32 weights (grad: RSDFT_LPC_NWEIGHTS
 * values, host).  loss/grad may be NULL. */
int rsdft_gpu_lpc_loss_grad(const float* x, const float* t, int nb, int n, int margin,
                            double* loss, float* grad, int mem);
/* Empty device training set for `capacity` pairs of patch^3 points. */
int rsdft_gpu_lpc_dataset(int capacity, int patch);
/* Append up to npatch pairs cut (periodic, random corners, random bands) from the resident
 * bands of (k, s): input = the CG gradient -2(H psi - E psi) scaled to unit RMS; target =
 * sigma (T + sigma)^-1 of it, T the finite-difference kinetic operator, by `iters` CG steps.
 * added receives the pairs stored. */
int rsdft_gpu_lpc_harvest(int k, int s, int npatch, double sigma, int iters,
                          unsigned long long seed, int* added);
/* Host copy of harvested pairs [first, first+count); x or t may be NULL. */
int rsdft_gpu_lpc_dataset_get(int first, int count, float* x, float* t);
/* Append count host pairs (patch^3 each) to the training set; added receives the pairs stored. */
int rsdft_gpu_lpc_dataset_add(const float* x, const float* t, int count, int* added);
/* Adam training on the harvested set (MSE on the patch interior); losses[epoch] (host, may be
 * NULL) receives the mean batch loss of each epoch. */
int rsdft_gpu_lpc_train(int margin, int epochs, int batch, double lr, unsigned long long seed,
                        double* losses);
/* The preconditioner on full periodic FP32 bands of the context grid: pg = rms(g) f(g/rms(g)). */
int rsdft_gpu_lpc_precond_f(const float* g, float* pg, int nb, int mem);
/* How the preconditioner (in CG and in rsdft_gpu_lpc_precond_f) evaluates the network: 0 (the
 * default) runs the two 16 -> 16 layers on the tensor cores with BF16 activations and FP32
 * accumulation, 1 runs all layers on CUDA cores with FP32 activations. */
int rsdft_gpu_lpc_inference(int mode);
/* ready: weights loaded; pc_in_use: the PC mode CG uses now; fallbacks: learned-to-plain
 * switches so far; dataset: harvested pairs.  Any output may be NULL. */
int rsdft_gpu_lpc_status(int* ready, int* pc_in_use, int* fallbacks, int* dataset);

/* ---- measurement ---- */
/* Per-kernel CUDA-event timing of the library's own launches: 0 off (the default), 1 every
 * kernel family, 2 the hpsi stencil only (two events per stencil launch and no host
 * synchronisation, so a timed solve is not slowed by it). */
int rsdft_gpu_profile(int on);
/* total device time (ms), launch count, algorithmic bytes and flops recorded for kernel
 * family `name` ("hpsi_stencil", "nl_gather", "gemm", "cg", "pc", ...); any output may be NULL.
 * "stencil_tune_r1" / "stencil_tune_r2" ("stencil64_..." for FP64) give the last autotuning
 * time of each stencil variant (rows per thread). */
int rsdft_gpu_profile_get(const char* name, double* total_ms, long long* launches, double* bytes,
                          double* flops);
/* Launch count of all library kernels since init (for launch accounting). */
long long rsdft_gpu_kernel_launches(void);
/* Diagnostic: the split-BF16 tensor-core GEMM against cuBLAS DGEMM on the same FP32 inputs.
 * op 0: C = A B^T (A: m x k, B: n x k); op 1: X <- X V (X: m bands x k points, V: m x m);
 * op 2 (n == m): the fused overlap/Hsub form [A A^T | A B^T] as the sweep computes it.
 * err receives max|x3 - dgemm| / max|dgemm|.  No counterpart in the reference. */
int rsdft_gpu_selftest_gemm(int m, int n, long long k, int op, double* err);
/* BF16 terms per FP32 value in the mixed-precision tensor-core contractions (2 or 3 each):
 * overlap_terms for S = dV Psi^T Psi and Hsub = dV Psi^T H Psi, rotation_terms for
 * Psi <- Psi V.  Three terms (the default for both) keep about FP32 accuracy per product; two
 * keep about 2^-16.  Two-term overlaps converge on small grids but leave the largest band
 * residual of the 128^3 / 2048-band problem wandering between 1e-7 and 1e-4; two-term rotations
 * stall the residual near 5e-9.  No counterpart in the reference. */
int rsdft_gpu_set_gemm_terms(int overlap_terms, int rotation_terms);
/* Precision schedule of rsdft_gpu_sweep (mixed precision): the Gram-Schmidt / subspace overlap and
 * Hsub contractions use two BF16 terms while CG's largest residual of the (k, s) in that sweep
 * is above res_sm, the band rotation while it is above res_rot; below, the terms set by
 * rsdft_gpu_set_gemm_terms.  0 switches a threshold off; the defaults are res_sm = 1e-2 and
 * res_rot = 1e-4 (the two-term noise, about 2^-16 relative per product, stays well below the
 * residuals of those sweeps).  No counterpart in the reference (one precision per build). */
int rsdft_gpu_set_gemm_schedule(double res_sm, double res_rot);
/* Tiling of the three-term tensor-core contractions, flags (default 7): bit 0 set, 128 x 256
 * output tiles over K blocks of 32 (else 128 x 128 over 64); bit 1 set, the overlap S of the
 * fused overlap/Hsub contraction is formed by the tiles reaching its upper triangle only (its
 * two triangles hold the same products), and with bit 3 also set Hsub the same way (the rest
 * mirrored; else both triangles, averaged); bit 2 set, the band rotation in plain form X C, else
 * in the update form X + X (C - I).  Measurement knob; no counterpart in the reference. */
int rsdft_gpu_set_gemm_tile(int flags);
/* Diagnostic: polls a bounded wait of the real build's hpsi stencil makes before it gives up
 * (0: it gives up at once; < 0: the default).  A wait that gives up ends the launch with
 * RSDFT_ERR_TIMEOUT from the entry that reads the device status word; the kernel first lets its
 * own bulk copies land, so the context stays usable.  Lets a test take the timeout path without
 * any GPU fault.  No counterpart in the reference. */
int rsdft_gpu_set_wait_polls(int polls);
/* Where the real build's hpsi adds the nonlocal term: 0 (default) a scatter kernel after the
 * stencil (one read-modify-write per covered point and band), 1 inside the streaming stencil
 * (records staged per plane).  Measurement knob; no counterpart in the reference. */
int rsdft_gpu_set_nl_form(int fused);
/* Real build's hpsi stencil: 0 (default) stages each plane's V_loc rows in shared memory with
 * the psi rows, 1 the consumer threads read them from global memory (L2-resident), which leaves
 * shared memory to more psi planes in flight.  Measurement knob; no counterpart in the
 * reference. */
int rsdft_gpu_set_stencil_form(int vloc_global);

#ifdef __cplusplus
}
#endif
#endif /* RSDFT_B200_H */
