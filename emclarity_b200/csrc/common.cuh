// common.cuh -- status handling, twiddle tables and small host helpers shared by
// every translation unit of libemc_b200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <cstring>
#include <string>

#include "../../include/emc_b200.h"
#include "fft.cuh"

namespace emc {

// Per-thread last error text (returned by emc_last_error()).
void set_error(const char* fmt, ...);

#define EMC_CHECK_ARG(cond, ...)            \
  do {                                      \
    if (!(cond)) {                          \
      ::emc::set_error(__VA_ARGS__);        \
      return EMC_E_ARG;                     \
    }                                       \
  } while (0)

#define EMC_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess) {                                                                    \
      ::emc::set_error("%s:%d: %s -> %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e));   \
      return _e == cudaErrorMemoryAllocation ? EMC_E_OOM : EMC_E_CUDA;                          \
    }                                                                                           \
  } while (0)

#define EMC_LAUNCH_CHECK() EMC_CUDA(cudaGetLastError())

#define EMC_TRY(expr)                 \
  do {                                \
    emc_status _s = (expr);           \
    if (_s != EMC_OK) return _s;      \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// True for the FFT edge lengths compiled into this library.
inline bool fft_length_supported(int n) {
  switch (n) {
    case 1: case 2: case 3: case 4: case 6: case 8: case 12: case 16: case 24: case 32: case 48:
    case 64: case 96: case 128: case 192: case 256: case 384: case 512:
      return true;
    default:
      return false;
  }
}

// Device twiddle table exp(-2 pi i m / L), m in [0, L), for every supported L,
// built once per device on first use (double precision on the host, rounded to float).
const float2* device_twiddles(int L);  // returns nullptr on failure (error text set)

// Device-side number of SMs (cached per device).
int device_sm_count();

}  // namespace emc
