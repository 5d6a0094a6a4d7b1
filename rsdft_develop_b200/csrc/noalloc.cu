// hamiltonian without device allocation.
//
// Some callers of the library cannot let it call cudaMalloc: a host code that reserves the
// whole device memory pool at start-up and forbids later allocations, a caller that drives
// the GPU from inside another framework's memory pool or stream capture, or a tight loop in
// which cudaMalloc's implicit device synchronisation would stall the pipeline.  This entry
// applies H to caller-owned device blocks and takes the only scratch it needs -- the
// nonlocal coefficient rows c_b[atom, projector] -- from a fixed array in device memory that
// is part of the library image instead of from the allocator.
#include "ctx.cuh"

namespace rsdft {

// Capacity of the scratch: nb * (atoms * projectors-per-atom, padded) coefficients per call.
constexpr size_t kNoAllocScratch = 1u << 19;  // 524288 doubles = 4 MiB per device

// Lives in every GPU that loads the library, until the process exits.  In host code the name
// is only a host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

static double* g_scratch_addr[64] = {nullptr};

// Resolve the device address of the scratch array for the current device (once per device).
static int scratch_address(double** out) {
  int dev = 0;
  RS_CUDA(cudaGetDevice(&dev));
  RS_CHECK(dev >= 0 && dev < 64, RSDFT_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    RS_CHECK(e == cudaSuccess && p != nullptr, RSDFT_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
             cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_hamiltonian_noalloc_d(int k, int s, const double* tpsi, double* htpsi, int ld, int nb) {
  Ctx* c = ctx();
  RS_CHECK(c != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");
  RS_CHECK(!c->cplx, RSDFT_ERR_STATE, "real entry on a complex16 context");
  RS_CHECK(k >= 1 && k <= c->p.nk && s >= 1 && s <= c->p.nspin, RSDFT_ERR_ARG, "(k,s)=(%d,%d) out of range", k, s);
  RS_CHECK(tpsi && htpsi && (size_t)ld >= c->ng && nb >= 0, RSDFT_ERR_ARG, "bad hamiltonian arguments");
  if (nb == 0) return 0;
  const size_t need = (size_t)nb * (size_t)c->nl.ngroups * (size_t)c->nl.pg;
  RS_CHECK(c->nl.nproj == 0 || need <= kNoAllocScratch, RSDFT_ERR_ARG,
           "hamiltonian_noalloc: %d bands x %d projector slots = %zu coefficients exceed the fixed scratch of %zu; "
           "call with fewer bands per block",
           nb, c->nl.ngroups * c->nl.pg, need, kNoAllocScratch);
  double* scratch = nullptr;
  RS_TRY(scratch_address(&scratch));
  return hpsi_real_scratch<double>(*c, k - 1, s - 1, tpsi, htpsi, (size_t)ld, nb, scratch, kNoAllocScratch);
}
