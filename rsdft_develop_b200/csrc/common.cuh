// Shared definitions for the RSDFT band-update library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuComplex.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rsdft_b200.h"

namespace rsdft {

// ---------------------------------------------------------------------------
// error handling: every C entry returns an int status; the message is kept.
// ---------------------------------------------------------------------------
void set_error(int code, const char* fmt, ...);
int last_code();

#define RS_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess) {                                                       \
      rsdft::set_error(RSDFT_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,   \
                       cudaGetErrorString(e_));                                    \
      return RSDFT_ERR_CUDA;                                                       \
    }                                                                              \
  } while (0)

#define RS_CHECK(cond, code, ...)                     \
  do {                                                \
    if (!(cond)) {                                    \
      rsdft::set_error((code), __VA_ARGS__);          \
      return (code);                                  \
    }                                                 \
  } while (0)

#define RS_TRY(expr)               \
  do {                             \
    int s_ = (expr);               \
    if (s_ != 0) return s_;        \
  } while (0)

// device status word bits (written by kernels whose bounded waits time out)
enum : unsigned { DEV_OK = 0u, DEV_WAIT_TIMEOUT = 1u, DEV_BAD_INDEX = 2u };

constexpr int MDMAX = 12;

// Stencil coefficients passed by value to kernels.
struct StencilCoef {
  double clap[3][MDMAX];   // coef_lap(d, m), m = 1..md
  double cnab[3][MDMAX];   // coef_nabk(d, m, k) (complex path)
  double c0;               // coef_lap0 + const_k2
};

// ---------------------------------------------------------------------------
// simple device buffer
// ---------------------------------------------------------------------------
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  int ensure(size_t nbytes) {
    if (nbytes <= bytes && p) return 0;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (nbytes == 0) return 0;
    cudaError_t e = cudaMalloc(&p, nbytes);
    if (e != cudaSuccess) {
      set_error(RSDFT_ERR_OOM, "cudaMalloc(%zu) failed: %s", nbytes, cudaGetErrorString(e));
      p = nullptr;
      return RSDFT_ERR_OOM;
    }
    bytes = nbytes;
    return 0;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
};

}  // namespace rsdft
