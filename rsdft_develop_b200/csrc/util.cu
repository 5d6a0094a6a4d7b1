// Small utility kernels: seeded initial wavefunctions and precision conversion.
#include "ctx.cuh"

namespace rsdft {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Irwin-Hall(12) - 6 per element; exact double arithmetic (see rsdft_b200.h).
template <typename T>
__global__ void k_random_wf(T* psi, unsigned long long ng, unsigned long long nb, int ncomp, uint64_t seed,
                            uint64_t k0) {
  const unsigned long long n = ng * nb * (unsigned long long)ncomp;
  for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < n;
       t += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long comp = t % ncomp;
    const unsigned long long rest = t / ncomp;
    const unsigned long long grid = rest % ng;
    const unsigned long long band = rest / ng;
    const uint64_t e = ((k0 * (1ull << 20) + band) * ng + grid) * 2ull + comp;
    const uint64_t base = seed * (1ull << 40) + e * 12ull;
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 12; ++q) acc = __dadd_rn(acc, (double)(splitmix64(base + (uint64_t)q) >> 11) * 0x1.0p-53);
    psi[t] = (T)(acc - 6.0);
  }
}

int random_wf(Ctx& c, int k, int s, uint64_t seed) {
  (void)s;
  WaveFns& w = c.wfn(k, s);
  const unsigned long long nb = (unsigned long long)c.kp[k].nband;
  const int ncomp = c.cplx ? 2 : 1;
  if (c.mixed)
    k_random_wf<float><<<4 * 148, 256, 0, c.stream>>>(w.psi.as<float>(), c.ng, nb, ncomp, seed, (uint64_t)k);
  else
    k_random_wf<double><<<4 * 148, 256, 0, c.stream>>>(w.psi.as<double>(), c.ng, nb, ncomp, seed, (uint64_t)k);
  c.launches++;
  return check_launch("random_wf");
}

__global__ void k_d2f(const double* __restrict__ s, float* __restrict__ d, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    d[i] = (float)s[i];
}
__global__ void k_f2d(const float* __restrict__ s, double* __restrict__ d, unsigned long long n) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    d[i] = (double)s[i];
}

int convert_d2f(Ctx& c, const double* src, float* dst, size_t n) {
  if (n == 0) return 0;
  k_d2f<<<8 * 148, 256, 0, c.stream>>>(src, dst, n);
  c.launches++;
  return check_launch("d2f");
}
int convert_f2d(Ctx& c, const float* src, double* dst, size_t n) {
  if (n == 0) return 0;
  k_f2d<<<8 * 148, 256, 0, c.stream>>>(src, dst, n);
  c.launches++;
  return check_launch("f2d");
}

}  // namespace rsdft
