// C ABI entry points, context management and operator set-up.
#include <cstdarg>
#include <cstring>
#include <cmath>
#include <unordered_map>

#include "ctx.cuh"

namespace rsdft {

static Ctx* g_ctx = nullptr;
static int g_code = 0;
static char g_msg[1024] = "";

void set_error(int code, const char* fmt, ...) {
  g_code = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}
int last_code() { return g_code; }
Ctx* ctx() { return g_ctx; }

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(RSDFT_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
    return RSDFT_ERR_CUDA;
  }
  return 0;
}

// ---- profiling ----
static cudaEvent_t take_event(Ctx& c) {
  if (!c.event_pool.empty()) {
    cudaEvent_t e = c.event_pool.back();
    c.event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
ProfScope::ProfScope(Ctx& c_, const char* n, double bytes_, double flops_)
    : c(c_), name(n), bytes(bytes_), flops(flops_) {
  if (!c.profiling || (c.profiling == 2 && std::strcmp(n, "hpsi_stencil") != 0)) return;
  e0 = take_event(c);
  e1 = take_event(c);
  cudaEventRecord(e0, c.stream);
}
ProfScope::~ProfScope() {
  if (!c.profiling || !e0) return;
  cudaEventRecord(e1, c.stream);
  c.pending.push_back({std::string(name), e0, e1, bytes, flops});
  if (c.pending.size() > 4096) prof_flush(c);
}
void prof_flush(Ctx& c) {
  if (c.pending.empty()) return;
  cudaStreamSynchronize(c.stream);
  for (auto& pe : c.pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, pe.e0, pe.e1);
    ProfEntry& e = c.prof[pe.name];
    e.ms += ms;
    e.launches += 1;
    e.bytes += pe.bytes;
    e.flops += pe.flops;
    c.event_pool.push_back(pe.e0);
    c.event_pool.push_back(pe.e1);
  }
  c.pending.clear();
}

// ---- device status word ----
static int check_status(Ctx& c) {
  unsigned h = 0;
  RS_CUDA(cudaMemcpyAsync(&h, c.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  if (h & DEV_WAIT_TIMEOUT) {
    unsigned z = 0;
    cudaMemcpy(c.d_status, &z, sizeof(unsigned), cudaMemcpyHostToDevice);
    set_error(RSDFT_ERR_TIMEOUT, "a bounded device-side wait timed out (status 0x%x)", h);
    return RSDFT_ERR_TIMEOUT;
  }
  return 0;
}

// ---- nonlocal tables ----
static int build_nonlocal(Ctx& c, int nzlma, int maxmjj, const int* mjj, const int* jjp, const int* amap,
                          int npair, const int* pairs, const double* dij) {
  NonlocalTables& nl = c.nl;
  nl = NonlocalTables();
  nl.nproj = nzlma;
  nl.maxmjj = maxmjj;
  if (nzlma == 0) return 0;
  nl.h_mjj.assign(mjj, mjj + nzlma);
  nl.h_jjp.assign(jjp, jjp + (size_t)nzlma * maxmjj);
  // groups = atoms in order of first appearance
  std::unordered_map<int, int> gid;
  std::vector<std::vector<int>> members;
  for (int p = 0; p < nzlma; ++p) {
    RS_CHECK(mjj[p] >= 0 && mjj[p] <= maxmjj, RSDFT_ERR_ARG, "MJJ(%d)=%d out of range", p + 1, mjj[p]);
    auto it = gid.find(amap[p]);
    if (it == gid.end()) {
      gid[amap[p]] = (int)members.size();
      members.push_back({p});
    } else {
      members[it->second].push_back(p);
    }
  }
  nl.ngroups = (int)members.size();
  int pmax = 0;
  for (auto& m : members) pmax = std::max(pmax, (int)m.size());
  nl.pg = pmax <= 1 ? 1 : pmax <= 4 ? 4 : pmax <= 9 ? 9 : pmax <= 16 ? 16 : 0;
  RS_CHECK(nl.pg > 0, RSDFT_ERR_UNSUPPORTED, "%d projectors on one atom (max 16)", pmax);
  const int PG = nl.pg;
  std::vector<int> proj_group(nzlma), proj_slot(nzlma);
  for (int g = 0; g < nl.ngroups; ++g)
    for (int i = 0; i < (int)members[g].size(); ++i) {
      proj_group[members[g][i]] = g;
      proj_slot[members[g][i]] = i;
    }
  // footprint union per group, first-occurrence order
  nl.h_gofs.assign(nl.ngroups + 1, 0);
  std::vector<int> gjj;
  nl.h_slot.assign((size_t)nzlma * maxmjj, -1);
  for (int g = 0; g < nl.ngroups; ++g) {
    std::unordered_map<int, int> slot;
    for (int p : members[g])
      for (int j = 0; j < mjj[p]; ++j) {
        const int pt = jjp[(size_t)p * maxmjj + j] - 1;
        RS_CHECK(pt >= 0 && (size_t)pt < c.ng, RSDFT_ERR_ARG, "JJP(%d,%d)=%d outside the grid", j + 1, p + 1,
                 pt + 1);
        auto it = slot.find(pt);
        int sl;
        if (it == slot.end()) {
          sl = (int)slot.size();
          slot[pt] = sl;
          gjj.push_back(pt);
        } else {
          sl = it->second;
        }
        nl.h_slot[(size_t)p * maxmjj + j] = nl.h_gofs[g] + sl;
      }
    nl.h_gofs[g + 1] = (int)gjj.size();
  }
  nl.ftotal = (int)gjj.size();
  nl.h_gplist.assign((size_t)nl.ngroups * PG, -1);
  for (int g = 0; g < nl.ngroups; ++g)
    for (int i = 0; i < (int)members[g].size(); ++i) nl.h_gplist[(size_t)g * PG + i] = members[g][i];
  // per-group dense coupling from the pair list
  std::vector<double> D((size_t)nl.ngroups * PG * PG, 0.0);
  for (int m = 0; m < npair; ++m) {
    const int l1 = pairs[2 * m] - 1, l2 = pairs[2 * m + 1] - 1;
    RS_CHECK(l1 >= 0 && l1 < nzlma && l2 >= 0 && l2 < nzlma, RSDFT_ERR_ARG, "nzqr_pair(:,%d) out of range", m + 1);
    RS_CHECK(proj_group[l1] == proj_group[l2], RSDFT_ERR_ARG,
             "nzqr_pair(:,%d) couples projectors of different atoms", m + 1);
    const int g = proj_group[l1];
    D[((size_t)g * PG + proj_slot[l1]) * PG + proj_slot[l2]] += dij[m];
  }
  // scatter records: one per (group, footprint point), sorted by grid point (stable counting sort)
  const int nrec = nl.ftotal;
  std::vector<int> cnt(c.ng + 1, 0), fslot_group(nrec);
  for (int g = 0; g < nl.ngroups; ++g)
    for (int f = nl.h_gofs[g]; f < nl.h_gofs[g + 1]; ++f) {
      cnt[gjj[f] + 1]++;
      fslot_group[f] = g;
    }
  std::vector<int> rowptr(c.ng + 16, 0);
  for (size_t i = 0; i < c.ng; ++i) rowptr[i + 1] = rowptr[i] + cnt[i + 1];
  for (size_t i = c.ng + 1; i < rowptr.size(); ++i) rowptr[i] = rowptr[c.ng];
  std::vector<int> fill(rowptr.begin(), rowptr.begin() + c.ng), rpt(nrec), rg(nrec);
  nl.h_rec_src.assign(nrec, 0);
  for (int f = 0; f < nrec; ++f) {
    const int e = fill[gjj[f]]++;
    rpt[e] = gjj[f];
    rg[e] = fslot_group[f];
    nl.h_rec_src[e] = f;
  }
  nl.nrec = nrec;
  RS_TRY(nl.gofs.ensure(nl.h_gofs.size() * sizeof(int)));
  RS_TRY(nl.gjj.ensure(std::max<size_t>(1, gjj.size()) * sizeof(int)));
  RS_TRY(nl.gplist.ensure(nl.h_gplist.size() * sizeof(int)));
  RS_TRY(nl.gD.ensure(D.size() * sizeof(double)));
  RS_TRY(nl.rec_rowptr.ensure(rowptr.size() * sizeof(int)));
  // record tables carry kRecPad spare records: the stencil's bulk copies round segments out to 4
  RS_TRY(nl.rec_pt.ensure((size_t)(nrec + kRecPad) * sizeof(int)));
  RS_TRY(nl.rec_g.ensure((size_t)(nrec + kRecPad) * sizeof(int)));
  RS_CUDA(cudaMemset(nl.rec_pt.p, 0, (size_t)(nrec + kRecPad) * sizeof(int)));
  RS_CUDA(cudaMemset(nl.rec_g.p, 0, (size_t)(nrec + kRecPad) * sizeof(int)));
  RS_CUDA(cudaMemcpy(nl.gofs.p, nl.h_gofs.data(), nl.h_gofs.size() * sizeof(int), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.gjj.p, gjj.data(), gjj.size() * sizeof(int), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.gplist.p, nl.h_gplist.data(), nl.h_gplist.size() * sizeof(int), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.gD.p, D.data(), D.size() * sizeof(double), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.rec_rowptr.p, rowptr.data(), rowptr.size() * sizeof(int), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.rec_pt.p, rpt.data(), nrec * sizeof(int), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(nl.rec_g.p, rg.data(), nrec * sizeof(int), cudaMemcpyHostToDevice));
  {  // covered grid points (the nonlocal scatter's work list)
    std::vector<int> cov;
    for (size_t i = 0; i < c.ng; ++i)
      if (rowptr[i + 1] > rowptr[i]) cov.push_back((int)i);
    nl.ncov = (int)cov.size();
    RS_TRY(nl.cov.ensure(std::max<size_t>(1, cov.size()) * sizeof(int)));
    if (!cov.empty())
      RS_CUDA(cudaMemcpy(nl.cov.p, cov.data(), cov.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  nl.perk.assign(c.p.nk, NonlocalTables::PerK());
  nl.h_rowptr.swap(rowptr);
  nl.seg_max.clear();
  return 0;
}

// uvk: real [nzlma][maxmjj] or interleaved complex [nzlma][maxmjj][2]
static int set_uvk(Ctx& c, int k, const double* uvk, bool cplx) {
  NonlocalTables& nl = c.nl;
  RS_CHECK(nl.nproj > 0, RSDFT_ERR_STATE, "set_projectors must precede set_uvk");
  const int PG = nl.pg, nc = cplx ? 2 : 1;
  std::vector<double> gw((size_t)nl.ftotal * PG * nc, 0.0), sw((size_t)nl.ftotal * PG * nc, 0.0),
      ru((size_t)(nl.nrec + kRecPad) * PG * nc, 0.0);
  std::vector<int> pslot(nl.nproj, 0);
  for (int g = 0; g < nl.ngroups; ++g)
    for (int i = 0; i < PG; ++i) {
      const int p = nl.h_gplist[(size_t)g * PG + i];
      if (p >= 0) pslot[p] = i;
    }
  for (int p = 0; p < nl.nproj; ++p)
    for (int j = 0; j < nl.h_mjj[p]; ++j) {
      const size_t e = (size_t)p * nl.maxmjj + j;
      const size_t w = ((size_t)nl.h_slot[e] * PG + pslot[p]) * nc;
      // gather weight conj(uVk) (src/ps_nloc_mr_module.f90:1290), scatter weight uVk (:1341);
      // duplicate grid points of one projector accumulate
      gw[w] += uvk[e * nc];
      sw[w] += uvk[e * nc];
      if (cplx) {
        gw[w + 1] -= uvk[e * nc + 1];
        sw[w + 1] += uvk[e * nc + 1];
      }
    }
  for (int r = 0; r < nl.nrec; ++r)
    for (int q = 0; q < PG * nc; ++q) ru[(size_t)r * PG * nc + q] = sw[(size_t)nl.h_rec_src[r] * PG * nc + q];
  NonlocalTables::PerK& pk = nl.perk[k];
  std::vector<float> gw32(gw.begin(), gw.end()), ru32(ru.begin(), ru.end());
  RS_TRY(pk.gw64.ensure(std::max<size_t>(1, gw.size()) * sizeof(double)));
  RS_TRY(pk.gw32.ensure(std::max<size_t>(1, gw.size()) * sizeof(float)));
  RS_TRY(pk.ru64.ensure(std::max<size_t>(1, ru.size()) * sizeof(double)));
  RS_TRY(pk.ru32.ensure(std::max<size_t>(1, ru.size()) * sizeof(float)));
  RS_CUDA(cudaMemcpy(pk.gw64.p, gw.data(), gw.size() * sizeof(double), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(pk.gw32.p, gw32.data(), gw32.size() * sizeof(float), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(pk.ru64.p, ru.data(), ru.size() * sizeof(double), cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(pk.ru32.p, ru32.data(), ru32.size() * sizeof(float), cudaMemcpyHostToDevice));
  pk.ready = true;
  return 0;
}

int nl_prepare_k(Ctx& c, int k) {
  RS_CHECK(c.nl.nproj == 0 || (k < (int)c.nl.perk.size() && c.nl.perk[k].ready), RSDFT_ERR_STATE,
           "uVk for k-point %d not set", k + 1);
  return 0;
}

static void destroy(Ctx* c) {
  if (!c) return;
  cudaStreamSynchronize(c->stream);
  for (auto& pe : c->pending) {
    cudaEventDestroy(pe.e0);
    cudaEventDestroy(pe.e1);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  DBuf* bufs[] = {&c->vloc64, &c->vloc32, &c->ws_coef, &c->ws_io_a, &c->ws_io_b, &c->ws_cg, &c->ws_red,
                  &c->ws_scal, &c->ws_dense, &c->ws_gram, &c->ws_hpsi, &c->ws_flag, &c->ws_rot, &c->ws_solver, &c->ws_info, &c->ws_gemm, &c->ws_out, &c->ws_f64,
                  &c->nl.gofs, &c->nl.gjj, &c->nl.gplist, &c->nl.gD, &c->nl.rec_rowptr, &c->nl.rec_pt, &c->nl.rec_g, &c->nl.cov};
  for (DBuf* b : bufs) b->release();
  for (auto& pk : c->nl.perk) {
    pk.gw64.release(); pk.gw32.release(); pk.ru64.release(); pk.ru32.release();
  }
  for (auto& w : c->wf) w.psi.release();
  scf_release(*c);
  if (c->d_status) cudaFree(c->d_status);
  if (c->cublas) cublasDestroy(c->cublas);
  if (c->syevj) cusolverDnDestroySyevjInfo(c->syevj);
  if (c->cusolver) cusolverDnDestroy(c->cusolver);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

template <typename T>
static int stage_in(Ctx& c, DBuf& buf, const T* src, size_t ld, int nb, int mem, const T** out) {
  if (mem == RSDFT_MEM_DEVICE) {
    *out = src;
    return 0;
  }
  RS_TRY(buf.ensure(sizeof(T) * ld * nb));
  RS_CUDA(cudaMemcpyAsync(buf.p, src, sizeof(T) * ld * nb, cudaMemcpyHostToDevice, c.stream));
  *out = buf.as<T>();
  return 0;
}

}  // namespace rsdft

using namespace rsdft;

#define REQUIRE_CTX() \
  RS_CHECK(g_ctx != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called")

template <typename T>
static int hamiltonian_entry(int k, int s, const T* tpsi, T* htpsi, int ld, int nb, int mem, bool cplx) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(cplx == c.cplx, RSDFT_ERR_STATE, "real/complex entry does not match the context");
  RS_CHECK(k >= 1 && k <= c.p.nk && s >= 1 && s <= c.p.nspin, RSDFT_ERR_ARG, "(k,s) out of range");
  RS_CHECK(tpsi && htpsi && ld > 0 && (size_t)ld >= c.ng && nb >= 0, RSDFT_ERR_ARG, "bad hamiltonian arguments");
  RS_CHECK(mem == RSDFT_MEM_HOST || mem == RSDFT_MEM_DEVICE, RSDFT_ERR_ARG, "bad memory space %d", mem);
  if (nb == 0) return 0;
  const int nc = cplx ? 2 : 1;
  const size_t ldn = (size_t)ld * nc;
  const T* din;
  RS_TRY(stage_in(c, c.ws_io_a, tpsi, ldn, nb, mem, &din));
  T* dout = htpsi;
  if (mem == RSDFT_MEM_HOST) {
    RS_TRY(c.ws_io_b.ensure(sizeof(T) * ldn * nb));
    dout = c.ws_io_b.as<T>();
  }
  if (cplx)
    RS_TRY(hpsi_cplx<T>(c, k - 1, s - 1, din, dout, ldn, nb));
  else
    RS_TRY(hpsi_real<T>(c, k - 1, s - 1, din, dout, ldn, nb));
  if (mem == RSDFT_MEM_HOST) {
    RS_CUDA(cudaMemcpyAsync(htpsi, dout, sizeof(T) * ldn * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
    return check_status(c);
  }
  return 0;
}



extern "C" {

const char* rsdft_gpu_last_error(void) { return g_msg; }

int rsdft_gpu_init(const rsdft_gpu_params* p) {
  RS_CHECK(p != nullptr, RSDFT_ERR_ARG, "params is NULL");
  if (g_ctx) {
    destroy(g_ctx);
    g_ctx = nullptr;
  }
  RS_CHECK(p->n1 > 0 && p->n2 > 0 && p->n3 > 0, RSDFT_ERR_ARG, "grid sizes must be positive");
  RS_CHECK(p->md >= 1 && p->md <= RSDFT_MDMAX, RSDFT_ERR_ARG, "Md=%d out of range", p->md);
  RS_CHECK(p->nk >= 1 && p->nspin >= 1 && p->mb >= 1, RSDFT_ERR_ARG, "nk, nspin, mb must be >= 1");
  RS_CHECK(p->precision == RSDFT_PREC_FP64 || p->precision == RSDFT_PREC_MIXED, RSDFT_ERR_ARG,
           "unknown precision mode %d", p->precision);
  RS_CHECK(p->pc_mode == RSDFT_PC_NONE || p->pc_mode == RSDFT_PC_HPRSDFT || p->pc_mode == RSDFT_PC_LEARNED,
           RSDFT_ERR_ARG, "unknown preconditioner mode %d", p->pc_mode);
  Ctx* c = new Ctx();
  c->p = *p;
  c->ng = (size_t)p->n1 * p->n2 * p->n3;
  c->pc_cur = p->pc_mode;
  c->cplx = p->is_complex != 0;
  {
    const char* e = getenv("RSDFT_EIG");
    c->eig_jacobi = e && std::strcmp(e, "syevj") == 0;
  }
  c->mixed = p->precision == RSDFT_PREC_MIXED;
  if (c->p.ncg <= 0) c->p.ncg = 3;
  if (c->p.mloop <= 0) c->p.mloop = 3;
  cudaGetDevice(&c->device);
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    set_error(RSDFT_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    delete c;
    return RSDFT_ERR_CUDA;
  }
  if (cublasCreate(&c->cublas) != CUBLAS_STATUS_SUCCESS || cusolverDnCreate(&c->cusolver) != CUSOLVER_STATUS_SUCCESS) {
    set_error(RSDFT_ERR_CUDA, "cuBLAS/cuSOLVER initialisation failed");
    destroy(c);
    return RSDFT_ERR_CUDA;
  }
  cublasSetStream(c->cublas, c->stream);
  cusolverDnSetStream(c->cusolver, c->stream);
  if (cudaMalloc(&c->d_status, sizeof(unsigned)) != cudaSuccess) {
    set_error(RSDFT_ERR_OOM, "status word allocation failed");
    destroy(c);
    return RSDFT_ERR_OOM;
  }
  cudaMemset(c->d_status, 0, sizeof(unsigned));
  c->kp.assign(p->nk, KPoint());
  for (auto& kk : c->kp) kk.nband = p->mb;
  c->vloc_set.assign(p->nspin, false);
  c->wf.resize((size_t)p->nk * p->nspin);
  c->nl.perk.assign(p->nk, NonlocalTables::PerK());
  g_ctx = c;
  return 0;
}

int rsdft_gpu_finalize(void) {
  lpc_release();
  destroy(g_ctx);
  g_ctx = nullptr;
  return 0;
}

int rsdft_gpu_get_stream(void** stream) {
  REQUIRE_CTX();
  RS_CHECK(stream != nullptr, RSDFT_ERR_ARG, "stream is NULL");
  *stream = (void*)g_ctx->stream;
  return 0;
}

int rsdft_gpu_synchronize(void) {
  REQUIRE_CTX();
  RS_CUDA(cudaStreamSynchronize(g_ctx->stream));
  return check_status(*g_ctx);
}

int rsdft_gpu_set_kpoint(int k, const double coef_nabk[3][RSDFT_MDMAX], double const_k2, int nband) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(k >= 1 && k <= c.p.nk, RSDFT_ERR_ARG, "k=%d out of range", k);
  RS_CHECK(nband >= 1 && nband <= c.p.mb, RSDFT_ERR_ARG, "nband=%d out of range (mb=%d)", nband, c.p.mb);
  KPoint& kp = c.kp[k - 1];
  if (coef_nabk) std::memcpy(kp.coef_nabk, coef_nabk, sizeof(kp.coef_nabk));
  kp.const_k2 = const_k2;
  kp.nband = nband;
  kp.set = true;
  return 0;
}

int rsdft_gpu_set_vloc(const double* vloc, int ml, int s) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(vloc != nullptr, RSDFT_ERR_ARG, "vloc is NULL");
  RS_CHECK((size_t)ml == c.ng, RSDFT_ERR_ARG, "ml=%d != grid size %zu", ml, c.ng);
  RS_CHECK(s >= 1 && s <= c.p.nspin, RSDFT_ERR_ARG, "s=%d out of range", s);
  for (size_t i = 0; i < c.ng; ++i)
    RS_CHECK(std::isfinite(vloc[i]), RSDFT_ERR_NUMERIC, "Vloc(%zu) is not finite", i + 1);
  RS_TRY(c.vloc64.ensure(sizeof(double) * c.ng * c.p.nspin));
  RS_TRY(c.vloc32.ensure(sizeof(float) * c.ng * c.p.nspin));
  std::vector<float> v32(vloc, vloc + c.ng);
  RS_CUDA(cudaMemcpy(c.vloc64.as<double>() + (size_t)(s - 1) * c.ng, vloc, sizeof(double) * c.ng,
                     cudaMemcpyHostToDevice));
  RS_CUDA(cudaMemcpy(c.vloc32.as<float>() + (size_t)(s - 1) * c.ng, v32.data(), sizeof(float) * c.ng,
                     cudaMemcpyHostToDevice));
  c.vloc_set[s - 1] = true;
  return 0;
}

int rsdft_gpu_set_projectors(int nzlma, int maxmjj, const int* mjj, const int* jjp, const int* amap, int npair,
                             const int* pairs, const double* dij00) {
  REQUIRE_CTX();
  RS_CHECK(nzlma >= 0 && maxmjj >= 0 && npair >= 0, RSDFT_ERR_ARG, "negative projector sizes");
  if (nzlma > 0)
    RS_CHECK(mjj && jjp && amap && (npair == 0 || (pairs && dij00)), RSDFT_ERR_ARG, "projector arrays are NULL");
  return build_nonlocal(*g_ctx, nzlma, maxmjj, mjj, jjp, amap, npair, pairs, dij00);
}

int rsdft_gpu_set_uvk_d(int k, const double* uvk) {
  REQUIRE_CTX();
  RS_CHECK(k >= 1 && k <= g_ctx->p.nk, RSDFT_ERR_ARG, "k=%d out of range", k);
  RS_CHECK(uvk != nullptr, RSDFT_ERR_ARG, "uvk is NULL");
  return set_uvk(*g_ctx, k - 1, uvk, false);
}

int rsdft_gpu_set_uvk_z(int k, const double* uvk) {
  REQUIRE_CTX();
  RS_CHECK(k >= 1 && k <= g_ctx->p.nk, RSDFT_ERR_ARG, "k=%d out of range", k);
  RS_CHECK(uvk != nullptr, RSDFT_ERR_ARG, "uvk is NULL");
  return set_uvk(*g_ctx, k - 1, uvk, true);
}

static int wf_slot(Ctx& c, int k, int s, WaveFns** w) {
  RS_CHECK(k >= 1 && k <= c.p.nk && s >= 1 && s <= c.p.nspin, RSDFT_ERR_ARG, "(k,s)=(%d,%d) out of range", k, s);
  *w = &c.wfn(k - 1, s - 1);
  return 0;
}

// Bands per chunk of the FP64 host <-> FP32 device transfers of the mixed-precision build
// (staging buffer of at most 1 GiB).
static int stage_bands(size_t n) { return (int)std::max<size_t>(1, ((size_t)1 << 30) / (sizeof(double) * n)); }

static int set_wf(int k, int s, const double* unk, int ld, int nb, bool cplx) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(cplx == c.cplx, RSDFT_ERR_STATE, "real/complex entry does not match the context");
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(unk != nullptr && (size_t)ld >= c.ng && nb == c.kp[k - 1].nband, RSDFT_ERR_ARG,
           "bad wavefunction block (ld=%d, nb=%d, nband=%d)", ld, nb, c.kp[k - 1].nband);
  const int nc = cplx ? 2 : 1;
  const size_t n = c.ng * nc;
  RS_TRY(w->psi.ensure(c.elem_bytes() * c.ng * (size_t)nb));
  if (!c.mixed) {
    RS_CUDA(cudaMemcpy2DAsync(w->psi.p, n * sizeof(double), unk, (size_t)ld * nc * sizeof(double),
                              n * sizeof(double), nb, cudaMemcpyHostToDevice, c.stream));
  } else {
    // FP64 host bands pass through a bounded device staging buffer in band chunks
    const int chunk = stage_bands(n);
    RS_TRY(c.ws_io_a.ensure(sizeof(double) * n * (size_t)std::min(chunk, nb)));
    for (int b0 = 0; b0 < nb; b0 += chunk) {
      const int cb = std::min(chunk, nb - b0);
      RS_CUDA(cudaMemcpy2DAsync(c.ws_io_a.p, n * sizeof(double), unk + (size_t)b0 * ld * nc,
                                (size_t)ld * nc * sizeof(double), n * sizeof(double), cb, cudaMemcpyHostToDevice,
                                c.stream));
      RS_TRY(convert_d2f(c, c.ws_io_a.as<double>(), w->psi.as<float>() + (size_t)b0 * n, n * cb));
    }
  }
  RS_CUDA(cudaStreamSynchronize(c.stream));
  w->valid = true;
  return 0;
}

static int get_wf(int k, int s, double* unk, int ld, int nb, bool cplx) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(cplx == c.cplx, RSDFT_ERR_STATE, "real/complex entry does not match the context");
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(w->valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k, s);
  RS_CHECK(unk != nullptr && (size_t)ld >= c.ng && nb >= 1 && nb <= c.kp[k - 1].nband, RSDFT_ERR_ARG,
           "bad wavefunction block");
  const int nc = cplx ? 2 : 1;
  const size_t n = c.ng * nc;
  if (!c.mixed) {
    RS_CUDA(cudaMemcpy2DAsync(unk, (size_t)ld * nc * sizeof(double), w->psi.p, n * sizeof(double),
                              n * sizeof(double), nb, cudaMemcpyDeviceToHost, c.stream));
  } else {
    const int chunk = stage_bands(n);
    RS_TRY(c.ws_io_a.ensure(sizeof(double) * n * (size_t)std::min(chunk, nb)));
    for (int b0 = 0; b0 < nb; b0 += chunk) {
      const int cb = std::min(chunk, nb - b0);
      RS_TRY(convert_f2d(c, w->psi.as<float>() + (size_t)b0 * n, c.ws_io_a.as<double>(), n * cb));
      RS_CUDA(cudaMemcpy2DAsync(unk + (size_t)b0 * ld * nc, (size_t)ld * nc * sizeof(double), c.ws_io_a.p,
                                n * sizeof(double), n * sizeof(double), cb, cudaMemcpyDeviceToHost, c.stream));
    }
  }
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return check_status(c);
}

int rsdft_gpu_set_wf_d(int k, int s, const double* unk, int ld, int nb) { return set_wf(k, s, unk, ld, nb, false); }
int rsdft_gpu_get_wf_d(int k, int s, double* unk, int ld, int nb) { return get_wf(k, s, unk, ld, nb, false); }
int rsdft_gpu_set_wf_z(int k, int s, const double* unk, int ld, int nb) { return set_wf(k, s, unk, ld, nb, true); }
int rsdft_gpu_get_wf_z(int k, int s, double* unk, int ld, int nb) { return get_wf(k, s, unk, ld, nb, true); }

int rsdft_gpu_random_wf(int k, int s, uint64_t seed) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_TRY(w->psi.ensure(c.elem_bytes() * c.ng * (size_t)c.kp[k - 1].nband));
  RS_TRY(random_wf(c, k - 1, s - 1, seed));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  w->valid = true;
  return 0;
}

int rsdft_gpu_hamiltonian_d(int k, int s, const double* tpsi, double* htpsi, int ld, int nb, int mem) {
  return hamiltonian_entry<double>(k, s, tpsi, htpsi, ld, nb, mem, false);
}
int rsdft_gpu_hamiltonian_f(int k, int s, const float* tpsi, float* htpsi, int ld, int nb, int mem) {
  return hamiltonian_entry<float>(k, s, tpsi, htpsi, ld, nb, mem, false);
}
int rsdft_gpu_hamiltonian_z(int k, int s, const double* tpsi, double* htpsi, int ld, int nb, int mem) {
  return hamiltonian_entry<double>(k, s, tpsi, htpsi, ld, nb, mem, true);
}
int rsdft_gpu_hamiltonian_c(int k, int s, const float* tpsi, float* htpsi, int ld, int nb, int mem) {
  return hamiltonian_entry<float>(k, s, tpsi, htpsi, ld, nb, mem, true);
}

}  // extern "C"

template <typename T>
static int precond_entry(int k, const T* gk, T* pgk, int ld, int nb, int mem) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(!c.cplx, RSDFT_ERR_STATE, "real entry on a complex16 context");
  RS_CHECK(k >= 1 && k <= c.p.nk, RSDFT_ERR_ARG, "k out of range");
  RS_CHECK(gk && pgk && (size_t)ld >= c.ng && nb >= 0, RSDFT_ERR_ARG, "bad precond arguments");
  if (nb == 0) return 0;
  const T* din;
  RS_TRY(stage_in(c, c.ws_io_a, gk, (size_t)ld, nb, mem, &din));
  T* dout = pgk;
  if (mem == RSDFT_MEM_HOST) {
    RS_TRY(c.ws_io_b.ensure(sizeof(T) * (size_t)ld * nb));
    dout = c.ws_io_b.as<T>();
  }
  RS_TRY(precond_real<T>(c, din, dout, (size_t)ld, nb));
  if (mem == RSDFT_MEM_HOST) {
    RS_CUDA(cudaMemcpyAsync(pgk, dout, sizeof(T) * (size_t)ld * nb, cudaMemcpyDeviceToHost, c.stream));
    RS_CUDA(cudaStreamSynchronize(c.stream));
  }
  return check_status(c);
}

extern "C" {

int rsdft_gpu_precond_d(int k, const double* gk, double* pgk, int ld, int nb, int mem) {
  return precond_entry<double>(k, gk, pgk, ld, nb, mem);
}
int rsdft_gpu_precond_f(int k, const float* gk, float* pgk, int ld, int nb, int mem) {
  return precond_entry<float>(k, gk, pgk, ld, nb, mem);
}

int rsdft_gpu_conjugate_gradient(int k, int s, double* esp, double* res) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(w->valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k, s);
  RS_TRY(cg_run(c, k - 1, s - 1, esp, res));
  return check_status(c);
}

int rsdft_gpu_gram_schmidt(int k, int s) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(w->valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k, s);
  RS_TRY(gs_run(c, k - 1, s - 1, 1));
  return check_status(c);
}

int rsdft_gpu_subspace_diag(int k, int s, double* esp) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(w->valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k, s);
  RS_TRY(sd_run(c, k - 1, s - 1, esp));
  return check_status(c);
}

int rsdft_gpu_residual(int k, int s, double* esp, double* res) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  WaveFns* w;
  RS_TRY(wf_slot(c, k, s, &w));
  RS_CHECK(w->valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k, s);
  const int nb = c.kp[k - 1].nband;
  RS_TRY(c.ws_out.ensure(sizeof(double) * 2 * (size_t)std::max(nb, 1) + 64));
  double* d = c.ws_out.as<double>();
  RS_TRY(residual_run(c, k - 1, s - 1, d, d + nb));
  if (esp) RS_CUDA(cudaMemcpyAsync(esp, d, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
  if (res) RS_CUDA(cudaMemcpyAsync(res, d + nb, sizeof(double) * nb, cudaMemcpyDeviceToHost, c.stream));
  RS_CUDA(cudaStreamSynchronize(c.stream));
  return check_status(c);
}

int rsdft_gpu_set_precision(int precision) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  RS_CHECK(precision == RSDFT_PREC_FP64 || precision == RSDFT_PREC_MIXED, RSDFT_ERR_ARG,
           "unknown precision mode %d", precision);
  const bool to_mixed = precision == RSDFT_PREC_MIXED;
  if (to_mixed == c.mixed) return 0;
  const size_t nc = c.cplx ? 2 : 1;
  for (int kk = 0; kk < c.p.nk; ++kk)
    for (int s = 0; s < c.p.nspin; ++s) {
      WaveFns& w = c.wfn(kk, s);
      if (!w.valid || !w.psi.p) continue;
      const size_t n = c.ng * nc * (size_t)c.kp[kk].nband;
      DBuf nb;
      RS_TRY(nb.ensure(n * (to_mixed ? sizeof(float) : sizeof(double))));
      if (to_mixed)
        RS_TRY(convert_d2f(c, w.psi.as<double>(), nb.as<float>(), n));
      else
        RS_TRY(convert_f2d(c, w.psi.as<float>(), nb.as<double>(), n));
      RS_CUDA(cudaStreamSynchronize(c.stream));
      w.psi.release();
      w.psi = nb;
    }
  c.mixed = to_mixed;
  c.p.precision = precision;
  c.cg_hx_ready = false;  // CG's H x array holds the other precision
  return check_status(c);
}

int rsdft_gpu_init_sweep(int mb_ref) {
  REQUIRE_CTX();
  RS_CHECK(mb_ref >= -1, RSDFT_ERR_ARG, "mb_ref must be >= -1");
  g_ctx->mb_ref = mb_ref;
  return 0;
}

int rsdft_gpu_set_sweep_check(int iconv_check) {
  REQUIRE_CTX();
  RS_CHECK(iconv_check == 0 || iconv_check == 2, RSDFT_ERR_ARG, "sweep check must be 0 or 2");
  g_ctx->sweep_check = iconv_check;
  return 0;
}

}  // extern "C"

// Bands 1..n of k-point k checked for convergence by rsdft_gpu_sweep
static int conv_bands(const Ctx& c, int k) {
  const int nb = c.kp[k].nband;
  if (c.mb_ref > 0) return std::min(c.mb_ref, nb);
  if (c.mb_ref < 0) return nb - nb / 8;
  return nb;
}

extern "C" {

int rsdft_gpu_sweep(int nsweep, double tol, int* iters, double* esp, double* res) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  const int nbmax = c.p.mb;
  std::vector<double> e((size_t)nbmax), r((size_t)nbmax);
  // learned-PC guard: every sweep is checked by the FP64 residual without preconditioning; when
  // it has not dropped below 0.9x its best value for 3 sweeps running, CG falls back to
  // precond_hprsdft for the rest of the run
  double best = 1e300;
  int stall = 0;
  int it = 0;
  std::vector<double> cg_res((size_t)nbmax);
  // sweep_check 2 (conv_check_2, src/sweep_module.f90:277-288): converged when no eigenvalue of
  // bands 1..mb_ref moved by tol or more in the sweep; esp0 holds the previous sweep's values
  const bool by_esp = c.sweep_check == 2;
  const size_t nall = (size_t)c.p.nspin * c.p.nk * nbmax;
  std::vector<double> esp_cur(by_esp ? nall : 0, 0.0), esp_old(by_esp ? nall : 0, 0.0);
  // esp0 of the first sweep: the Ritz values of the context's last sweep (the reference's esp
  // array keeps them across calc_sweep calls, e.g. from the previous k of the band trajectory)
  if (by_esp && c.esp_last.size() == nall) esp_old = c.esp_last;
  for (it = 1; it <= nsweep; ++it) {
    double rmax = 0.0, cg_rmax = 0.0, dmax = 0.0;
    for (int s = 0; s < c.p.nspin; ++s)
      for (int k = 0; k < c.p.nk; ++k) {
        RS_CHECK(c.wfn(k, s).valid, RSDFT_ERR_STATE, "no wavefunctions resident for (k,s)=(%d,%d)", k + 1, s + 1);
        RS_TRY(cg_run(c, k, s, nullptr, cg_res.data()));
        const int nconv = conv_bands(c, k);
        for (int n = 0; n < nconv; ++n) cg_rmax = std::max(cg_rmax, cg_res[n]);
        const size_t off = ((size_t)s * c.p.nk + k) * nbmax;
        // precision schedule (mixed precision): two BF16 terms in the contractions while CG's
        // residual of this (k, s) is above the threshold, then the configured terms
        const int t_sm = c.gemm_terms_sm, t_rot = c.gemm_terms_rot;
        double kmax = 0.0;
        for (int n = 0; n < nconv; ++n) kmax = std::max(kmax, cg_res[n]);
        if (c.sched_res_sm > 0.0 && kmax > c.sched_res_sm) c.gemm_terms_sm = 2;
        if (c.sched_res_rot > 0.0 && kmax > c.sched_res_rot) c.gemm_terms_rot = 2;
        if (c.gemm_terms_sm != t_sm || c.gemm_terms_rot != t_rot) c.sched_sweeps++;
        const int rc_g = gssd_run(c, k, s, by_esp ? esp_cur.data() + off : nullptr, true);
        c.gemm_terms_sm = t_sm;
        c.gemm_terms_rot = t_rot;
        RS_TRY(rc_g);
        if (by_esp) {
          for (int n = 0; n < nconv; ++n) dmax = std::max(dmax, std::fabs(esp_cur[off + n] - esp_old[off + n]));
        }
      }
    if (by_esp) {
      const bool done = tol > 0.0 && dmax < tol;
      if (done || it == nsweep) {
        for (int s = 0; s < c.p.nspin; ++s)
          for (int k = 0; k < c.p.nk; ++k) {
            const int nb = c.kp[k].nband;
            const size_t off = ((size_t)s * c.p.nk + k) * nbmax;
            RS_TRY(rsdft_gpu_residual(k + 1, s + 1, e.data(), r.data()));
            if (esp) std::memcpy(esp + off, e.data(), sizeof(double) * nb);
            if (res) std::memcpy(res + off, r.data(), sizeof(double) * nb);
          }
      }
      c.esp_last = esp_cur;
      if (done) break;
      esp_old.swap(esp_cur);
      continue;
    }
    // The FP64 check (an FP64 H x of every band) runs once CG's own residual of the bands it
    // returned is within kResGate x tol: before that the check cannot pass.  The learned-PC
    // guard checks every sweep.
    constexpr double kResGate = 30.0;
    const bool check_fp64 = tol > 0.0 && (cg_rmax <= kResGate * tol || pc_effective(c) == RSDFT_PC_LEARNED);
    if (check_fp64 || it == nsweep) {
      for (int s = 0; s < c.p.nspin; ++s)
        for (int k = 0; k < c.p.nk; ++k) {
          const int nb = c.kp[k].nband;
          RS_TRY(rsdft_gpu_residual(k + 1, s + 1, e.data(), r.data()));
          const int nconv = conv_bands(c, k);
          for (int n = 0; n < nconv; ++n) rmax = std::max(rmax, r[n]);
          const size_t off = ((size_t)s * c.p.nk + k) * nbmax;
          if (esp) std::memcpy(esp + off, e.data(), sizeof(double) * nb);
          if (res) std::memcpy(res + off, r.data(), sizeof(double) * nb);
        }
      if (pc_effective(c) == RSDFT_PC_LEARNED) {
        if (rmax < 0.9 * best) {
          best = rmax;
          stall = 0;
        } else if (++stall >= 3) {
          c.pc_cur = RSDFT_PC_HPRSDFT;
          c.lpc_fallbacks++;
        }
      }
      if (tol > 0.0 && rmax <= tol) break;
    }
  }
  if (iters) *iters = std::min(it, nsweep);
  return check_status(c);
}

int rsdft_gpu_profile(int on) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  prof_flush(c);
  RS_CHECK(on >= 0 && on <= 2, RSDFT_ERR_ARG, "profile mode must be 0, 1 or 2");
  c.profiling = on;
  if (on) c.prof.clear();
  return 0;
}

int rsdft_gpu_profile_get(const char* name, double* total_ms, long long* launches, double* bytes, double* flops) {
  REQUIRE_CTX();
  Ctx& c = *g_ctx;
  prof_flush(c);
  if (name && std::strcmp(name, "workspace_bytes") == 0) {
    if (total_ms) *total_ms = 0.0;
    if (launches) *launches = 0;
    if (bytes) *bytes = (double)c.workspace_bytes();
    if (flops) *flops = 0.0;
    return 0;
  }
  auto it = c.prof.find(name ? name : "");
  const bool f = it != c.prof.end();
  if (!f && name) {
    auto tt = c.tune_ms.find(name);
    if (tt != c.tune_ms.end()) {
      if (total_ms) *total_ms = tt->second;
      if (launches) *launches = 1;
      if (bytes) *bytes = 0.0;
      if (flops) *flops = 0.0;
      return 0;
    }
  }
  if (total_ms) *total_ms = f ? it->second.ms : 0.0;
  if (launches) *launches = f ? it->second.launches : 0;
  if (bytes) *bytes = f ? it->second.bytes : 0.0;
  if (flops) *flops = f ? it->second.flops : 0.0;
  return 0;
}

long long rsdft_gpu_kernel_launches(void) { return g_ctx ? g_ctx->launches : 0; }

int rsdft_gpu_selftest_gemm(int m, int n, long long k, int op, double* err) {
  REQUIRE_CTX();
  RS_CHECK(m > 0 && n > 0 && k > 0 && err && op >= 0 && op <= 2, RSDFT_ERR_ARG, "bad selftest arguments");
  RS_TRY(selftest_gemm(*g_ctx, m, n, k, op, op == 1 ? g_ctx->gemm_terms_rot : g_ctx->gemm_terms_sm, err));
  return check_status(*g_ctx);
}

int rsdft_gpu_set_pc_form(int form) {
  REQUIRE_CTX();
  RS_CHECK(form >= 0 && form <= 3, RSDFT_ERR_ARG, "preconditioner form must be 0, 1, 2 or 3");
  g_ctx->pc_sstep = form == 3 ? 1 : form;
  g_ctx->pc_direct = form == 3 ? 1 : 0;
  return 0;
}

int rsdft_gpu_set_stencil_form(int vloc_global) {
  REQUIRE_CTX();
  RS_CHECK(vloc_global == 0 || vloc_global == 1, RSDFT_ERR_ARG, "vloc_global must be 0 or 1");
  g_ctx->stencil_vloc_global = vloc_global;
  return 0;
}

int rsdft_gpu_set_nl_form(int fused) {
  REQUIRE_CTX();
  RS_CHECK(fused == 0 || fused == 1, RSDFT_ERR_ARG, "fused must be 0 or 1");
  g_ctx->nl_fused = fused;
  g_ctx->stencil_tune.clear();  // the stencil's best configuration depends on it
  return 0;
}

int rsdft_gpu_set_cggs(int iswitch) {
  REQUIRE_CTX();
  RS_CHECK(iswitch >= 0 && iswitch <= 2, RSDFT_ERR_ARG, "cggs switch must be 0, 1 or 2");
  g_ctx->cggs = iswitch;
  return 0;
}

int rsdft_gpu_set_wait_polls(int polls) {
  REQUIRE_CTX();
  g_ctx->wait_polls = polls < 0 ? -1 : polls;
  return 0;
}

int rsdft_gpu_set_gemm_tile(int flags) {
  REQUIRE_CTX();
  RS_CHECK(flags >= 0 && flags <= 15, RSDFT_ERR_ARG, "tile flags must be in 0..15");
  g_ctx->gemm_wide = flags & 1;
  g_ctx->gemm_tri = ((flags >> 1) & 1) ? (((flags >> 3) & 1) ? 2 : 1) : 0;
  g_ctx->rot_update = ((flags >> 2) & 1) ? 0 : 1;
  return 0;
}

int rsdft_gpu_set_gemm_terms(int overlap_terms, int rotation_terms) {
  REQUIRE_CTX();
  RS_CHECK((overlap_terms == 2 || overlap_terms == 3) && (rotation_terms == 2 || rotation_terms == 3), RSDFT_ERR_ARG,
           "split terms must be 2 or 3");
  g_ctx->gemm_terms_sm = overlap_terms;
  g_ctx->gemm_terms_rot = rotation_terms;
  return 0;
}

int rsdft_gpu_set_gemm_schedule(double res_sm, double res_rot) {
  REQUIRE_CTX();
  RS_CHECK(res_sm >= 0.0 && res_rot >= 0.0, RSDFT_ERR_ARG, "schedule thresholds must be >= 0");
  g_ctx->sched_res_sm = res_sm;
  g_ctx->sched_res_rot = res_rot;
  return 0;
}

}  // extern "C"
