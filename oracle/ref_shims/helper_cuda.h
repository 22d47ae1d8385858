// Test-infrastructure shim (oracle build only): the two error-check macros the
// reference sources expect from the CUDA samples' helper_cuda.h, which is not
// shipped with the toolkit. Written for this project; exits like the original.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#define checkCudaErrors(call)                                                  \
  do {                                                                         \
    cudaError_t rw_shim_err_ = (call);                                         \
    if (rw_shim_err_ != cudaSuccess) {                                         \
      std::fprintf(stderr, "CUDA error %d (%s) at %s:%d\n", (int)rw_shim_err_, \
                   cudaGetErrorString(rw_shim_err_), __FILE__, __LINE__);      \
      std::exit(EXIT_FAILURE);                                                 \
    }                                                                          \
  } while (0)

#define getLastCudaError(msg)                                                  \
  do {                                                                         \
    cudaError_t rw_shim_err_ = cudaGetLastError();                             \
    if (rw_shim_err_ != cudaSuccess) {                                         \
      std::fprintf(stderr, "%s: CUDA error %d (%s) at %s:%d\n", (msg),         \
                   (int)rw_shim_err_, cudaGetErrorString(rw_shim_err_),        \
                   __FILE__, __LINE__);                                        \
      std::exit(EXIT_FAILURE);                                                 \
    }                                                                          \
  } while (0)
