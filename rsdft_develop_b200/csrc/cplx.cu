// complex16 (k-point) build: hpsi, CG, GS and SD on interleaved complex arrays.
#include "ctx.cuh"

namespace rsdft {

template <typename T>
int hpsi_cplx(Ctx& c, int k, int s, const T* psi, T* hpsi, size_t ld, int nb) {
  (void)c; (void)k; (void)s; (void)psi; (void)hpsi; (void)ld; (void)nb;
  RS_CHECK(false, RSDFT_ERR_UNSUPPORTED, "complex16 hpsi not built yet");
}
template int hpsi_cplx<float>(Ctx&, int, int, const float*, float*, size_t, int);
template int hpsi_cplx<double>(Ctx&, int, int, const double*, double*, size_t, int);

}  // namespace rsdft
