// Library context: operator tables, resident wavefunctions and workspaces.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <algorithm>
#include <map>
#include <type_traits>
#include <string>

#include "common.cuh"

namespace rsdft {

constexpr int kRecPad = 8;  // spare records at the end of the scatter-record tables

// Nonlocal projectors grouped by atom (footprint union), for the gather kernel,
// plus the per-point CSR used by the scatter fused into the stencil kernel.
struct NonlocalTables {
  int nproj = 0;          // nzlma
  int ngroups = 0;        // atoms
  int pg = 0;             // padded projectors per group (1, 4, 9, 16)
  int ftotal = 0;         // total footprint entries over groups
  std::vector<int> h_gofs, h_gplist;         // host copies (group layout)
  DBuf gofs, gjj, gplist, gD;                // int / int / int[ngroups*PG] / double[ngroups*PG*PG]
  // scatter records: one per (group, footprint point), sorted by grid point
  DBuf rec_rowptr, rec_pt, rec_g;            // (ng+1 padded), (nrec), (nrec)
  int nrec = 0;
  // per k: gather weights conj(uVk) and scatter weights uVk, both [ftotal|nrec][PG] (T or T2)
  struct PerK {
    DBuf gw64, gw32;
    DBuf ru64, ru32;
    bool ready = false;
  };
  std::vector<PerK> perk;
  // host-side copies needed to build per-k tables
  std::vector<int> h_mjj, h_jjp;  // reference layout
  int maxmjj = 0;
  std::vector<int> h_slot;        // for each (lma, j): footprint slot in its group
  std::vector<int> h_rec_src;     // for each record: its footprint slot
  std::vector<int> h_rowptr;      // host copy of rec_rowptr
  DBuf cov;                       // grid points with at least one record, ascending
  int ncov = 0;
  std::map<int, int> seg_max;     // tile_y -> largest record segment of one (plane, y-tile)
};

struct KPoint {
  double coef_nabk[3][MDMAX] = {};
  double const_k2 = 0.0;
  int nband = 0;
  bool set = false;
};

struct WaveFns {
  DBuf psi;        // resident unk: FP64 (double / double2) or FP32 (float / float2)
  bool valid = false;
};

struct ProfEntry {
  double ms = 0.0;
  long long launches = 0;
  double bytes = 0.0;   // algorithmic bytes moved by the bracketed launches
  double flops = 0.0;   // algorithmic flops of the bracketed launches
};

// device state of the SCF pieces (scf.cu): density, potentials, Pulay history
struct ScfState {
  DBuf vion, rho, vh, vxc, occ, work, part, ones;
  DBuf xin, xou, xin_bak, xou_bak, xold_f, xold_g, h, f0, w;
  DBuf gga;                     // rsdft_gpu_xc_pbe: density, gradient, fluxes, potentials, partials
  bool have_rho = false, mixing = false, plans = false;
  int plan_f = 0, plan_b = 0;   // cuFFT handles (D2Z, Z2D)
  int mmix = 4, mmix_count = 0;
  double beta = 1.1, dif0 = 0.0;
};

struct Ctx {
  rsdft_gpu_params p{};
  size_t ng = 0;
  bool cplx = false;
  bool mixed = false;
  cudaStream_t stream = nullptr;
  int device = 0;                  // the CUDA device current at rsdft_gpu_init
  double* noalloc_scratch = nullptr;  // device address of the allocation-free entry's fixed array
  cublasHandle_t cublas = nullptr;
  cusolverDnHandle_t cusolver = nullptr;
  unsigned* d_status = nullptr;
  long long launches = 0;
  int mb_ref = 0;  // bands 1..mb_ref checked for convergence (0: all)
  int sweep_check = 0;  // rsdft_gpu_sweep convergence: 0 FP64 residual <= tol, 2 eigenvalue change < tol
  std::vector<double> esp_last;  // Ritz values of the last sweep (sweep_check 2), [s][k][band]
  bool eig_jacobi = false;          // subspace eigensolver: Jacobi (syevj) instead of syevd
  syevjInfo_t syevj = nullptr;

  ScfState scf;
  std::vector<KPoint> kp;
  DBuf vloc64, vloc32;             // [nspin][ng]
  std::vector<bool> vloc_set;
  NonlocalTables nl;
  std::vector<WaveFns> wf;         // [k][s]

  // workspaces
  DBuf ws_coef;                    // nonlocal coefficients [nb][nproj]
  DBuf ws_io_a, ws_io_b;           // staging for host-pointer hamiltonian calls
  DBuf ws_cg;                      // CG / PC block vectors
  DBuf ws_red;                     // reduction partials
  DBuf ws_scal;                    // per-band scalars (double)
  DBuf ws_dense;                   // M x M matrices
  DBuf ws_gram;                    // per-CTA partials of the small-band FP64 Gram matrices
  DBuf ws_hpsi;                    // H psi of all bands (nb x ng): CG's running H x, subspace diag
  DBuf ws_flag;                    // device counters (CG line-search rejections)
  bool cg_hx_ready = false;        // ws_hpsi holds H x of every band of (cg_hx_k, cg_hx_s) after CG
  int cg_hx_k = -1, cg_hx_s = -1;
  DBuf ws_rot;                     // rotation / GS temporaries
  DBuf ws_solver;                  // cusolver workspace
  DBuf ws_info;                    // cusolver info
  DBuf ws_gemm;                    // split-BF16 operands
  DBuf ws_out;                     // small per-band outputs (esp/res) handed to callers
  DBuf ws_f64;                     // FP64 copy of FP32-resident bands (mixed mode dense ops)
  DBuf vzero;                      // zero potential (kinetic-only operator)
  std::map<long long, int> stencil_tune;  // autotuned stencil variant (rows per thread) per shape
  std::map<std::string, double> tune_ms;   // last autotuning timings (reported by profile_get)
  int pc_cur = 0;                  // preconditioner in use by CG (pc_mode, or its fallback)
  int lpc_fallbacks = 0;           // sweeps-level switches from the learned to the plain PC
  int lpc_fp32 = 0;                // learned PC inference: 0 tensor cores (BF16 activations), 1 FP32 CUDA cores
  int gemm_terms_sm = 3;           // BF16 terms of the overlap / Hsub contractions (mixed precision)
  int gemm_terms_rot = 3;          // BF16 terms of the band rotations (mixed precision)
  double sched_res_sm = 1e-2;      // sweeps: 2 overlap/Hsub terms while CG's max residual > this (0: off)
  double sched_res_rot = 1e-4;     // sweeps: 2 rotation terms while CG's max residual > this (0: off)
  long long sched_sweeps = 0;      // (k, s) sweep steps run with reduced terms
  int pc_sstep = 1;                // FP32 precond_hprsdft: 1 s-step passes, 2 fused z-streamed s-step form
  int stencil_vloc_global = 0;     // real-build stencil: V_loc rows read from L2 instead of staged
  int pc_direct = 1;               // s-step passes: the last one forms the CG direction P (no PG, no k_make_p)
                                   // inside CG, 0 the recurrence form
  int gemm_wide = 1;               // three-term GEMM tiles 128 x 256 (K blocks of 32), else 128 x 128
  int gemm_tri = 1;                // S by upper-triangle tiles (1), S and Hsub (2), neither (0)
  int rot_update = 0;              // mixed rotation in update form X + X (C - I)
  int nl_fused = 0;                // nonlocal term inside the stencil (1) or by the scatter kernel after it (0)
  int wait_polls = -1;             // hpsi stencil's bounded waits: polls before giving up (-1: the default)
  int cggs = 0;                    // SWGS: 0 off, 1 cggs_1 (lower bands), 2 cggs_2 (all other bands)

  // profiling: 0 off, 1 every kernel family, 2 the hpsi stencil only (light enough for a timed run)
  int profiling = 0;
  std::map<std::string, ProfEntry> prof;
  struct Pending {
    std::string name;
    cudaEvent_t e0, e1;
    double bytes, flops;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;

  WaveFns& wfn(int k, int s) { return wf[(size_t)k * p.nspin + s]; }
  size_t workspace_bytes() const {  // device bytes of the context's growable workspaces
    return ws_coef.bytes + ws_io_a.bytes + ws_io_b.bytes + ws_cg.bytes + ws_red.bytes + ws_scal.bytes + ws_dense.bytes +
           ws_hpsi.bytes + ws_flag.bytes + ws_rot.bytes + ws_solver.bytes + ws_info.bytes + ws_gemm.bytes + ws_out.bytes +
           ws_f64.bytes + vzero.bytes;
  }
  size_t elem_bytes() const { return (mixed ? 4 : 8) * (cplx ? 2 : 1); }
};

Ctx* ctx();   // the process-wide context (null before init)

// profiling helpers: bracket a launch sequence with events on the library stream
struct ProfScope {
  Ctx& c;
  const char* name;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double bytes = 0.0, flops = 0.0;
  ProfScope(Ctx& c_, const char* n, double bytes_ = 0.0, double flops_ = 0.0);
  ~ProfScope();
};
void prof_flush(Ctx& c);

// error check after a launch
int check_launch(const char* what);

// ---- hpsi ----
template <typename T>
int hpsi_real(Ctx& c, int k, int s, const T* psi, T* hpsi, size_t ld, int nb);
template <typename T>
int hpsi_cplx(Ctx& c, int k, int s, const T* psi, T* hpsi, size_t ld, int nb);  // T = float / double (interleaved)
int nl_prepare_k(Ctx& c, int k);
template <typename T>
int hpsi_real_scratch(Ctx& c, int k, int s, const T* psi, T* hpsi, size_t ld, int nb, T* coef, size_t coef_cap);

int kinetic_shifted(Ctx& c, const float* x, float* y, size_t ld, int nb, double shift);

// ---- learned preconditioner (lpc.cu) ----
bool lpc_ready();
void lpc_release();
void scf_release(Ctx& c);
int lpc_apply(Ctx& c, const float* g, float* pg, int nb);
int pc_effective(const Ctx& c);

// ---- preconditioner / CG ----
int cg_run(Ctx& c, int k, int s, double* h_esp, double* h_res);
template <typename T>
int precond_real(Ctx& c, const T* g, T* pg, size_t ld, int nb);

// ---- dense ----
int gs_run(Ctx& c, int k, int s, int passes);
int sd_run(Ctx& c, int k, int s, double* h_esp);
int gssd_run(Ctx& c, int k, int s, double* h_esp, bool use_cg_hx);  // fused GS + SD of the sweep
int residual_run(Ctx& c, int k, int s, double* d_esp, double* d_res);

// ---- split-BF16 tensor-core GEMMs (gemm_x3.cu) ----
int gemm_tn_x3(Ctx& c, const float* A, long long lda, int M, const float* B, long long ldb, int N, long long K,
               double alpha, double* C, long long ldc, int swapB, int terms);
int gemm_tn2_x3(Ctx& c, const float* X, const float* Y, long long ld, int nb, long long K, double alpha, double* S,
                double* M, int terms);
int gemm_rotate_x3(Ctx& c, float* X, long long ldx, int nb, long long G, const double* V, int ldv, int terms,
                   bool add = false);
int selftest_gemm(Ctx& c, int m, int n, long long k, int op, int terms, double* err);
int gemm_tn_cat_x3(Ctx& c, const float* A, long long lda, int M, const float* const* B, const int* swap, int nparts,
                   long long ldb, int np, long long K, double alpha, double* const* Cp, long long ldc, int terms);
int gemm_rotate_cx3(Ctx& c, float* X, long long ldx, int nb, long long G, const double* Cz, int terms);

// ---- util ----
int random_wf(Ctx& c, int k, int s, uint64_t seed);
int convert_d2f(Ctx& c, const double* src, float* dst, size_t n);
int convert_f2d(Ctx& c, const float* src, double* dst, size_t n);

}  // namespace rsdft
