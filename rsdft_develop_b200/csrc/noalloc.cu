// hamiltonian without device allocation.
//
// Some callers of the library cannot let it call cudaMalloc: a host code that reserves the
// whole device memory pool at start-up and forbids later allocations, a caller that drives
// the GPU from inside another framework's memory pool, or a tight loop in which cudaMalloc's
// implicit device synchronisation would stall the pipeline.  This entry applies H to
// caller-owned device blocks and takes the only scratch it needs -- the nonlocal coefficient
// rows c_b[atom, projector] -- from a fixed array in device memory that is part of the library
// image instead of from the allocator.
#include "ctx.cuh"

namespace rsdft {

// Capacity of the scratch: nb * (atoms * projectors-per-atom, padded) coefficients per call.
constexpr size_t kNoAllocScratch = 1u << 19;  // 524288 doubles = 4 MiB per device

// Lives in every GPU that loads the library, until the process exits.  In host code the name
// is only a host-side stand-in; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

// Device address of the scratch array for the context's device, looked up by the first call
// of a context (with that device current) and kept in the context, so that a new context
// (after rsdft_gpu_finalize, or a device reset and rsdft_gpu_init) looks it up again.
static int scratch_address(Ctx& c, double** out) {
  int dev = -1;
  RS_CUDA(cudaGetDevice(&dev));
  RS_CHECK(dev == c.device, RSDFT_ERR_STATE,
           "hamiltonian_noalloc: device %d is current but the context was initialised on device %d", dev, c.device);
  if (!c.noalloc_scratch) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    RS_CHECK(e == cudaSuccess && p != nullptr, RSDFT_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
             cudaGetErrorString(e));
    c.noalloc_scratch = static_cast<double*>(p);
  }
  *out = c.noalloc_scratch;
  return 0;
}

}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_hamiltonian_noalloc_d(int k, int s, const double* tpsi, double* htpsi, int ld, int nb) {
  Ctx* c = ctx();
  RS_CHECK(c != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");
  RS_CHECK(!c->cplx, RSDFT_ERR_STATE, "real entry on a complex16 context");
  RS_CHECK(k >= 1 && k <= c->p.nk && s >= 1 && s <= c->p.nspin, RSDFT_ERR_ARG, "(k,s)=(%d,%d) out of range", k, s);
  RS_CHECK(tpsi && htpsi && ld > 0 && (size_t)ld >= c->ng && nb >= 0, RSDFT_ERR_ARG, "bad hamiltonian arguments");
  if (nb == 0) return 0;
  const size_t need = (size_t)nb * (size_t)c->nl.ngroups * (size_t)c->nl.pg;
  RS_CHECK(c->nl.nproj == 0 || need <= kNoAllocScratch, RSDFT_ERR_ARG,
           "hamiltonian_noalloc: %d bands x %d projector slots = %zu coefficients exceed the fixed scratch of %zu; "
           "call with fewer bands per block",
           nb, c->nl.ngroups * c->nl.pg, need, kNoAllocScratch);
  double* scratch = nullptr;
  RS_TRY(scratch_address(*c, &scratch));
  return hpsi_real_scratch<double>(*c, k - 1, s - 1, tpsi, htpsi, (size_t)ld, nb, scratch, kNoAllocScratch);
}
