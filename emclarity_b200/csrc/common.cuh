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

// FFT edge lengths compiled into this library: 2^a 3^b up to 512 used by the search plus the
// "nextBest" sizes of coordinates/BH_multi_iterator.m:3-5 (factors 5, 7, 13).
#define EMC_FOR_EACH_LENGTH(X) \
  X(2) X(3) X(4) X(6) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(72) X(80) X(84) X(90) X(96) \
  X(108) X(112) X(120) X(126) X(128) X(144) X(160) X(162) X(168) X(180) X(192) X(216) X(224) X(240) X(252) X(256) \
  X(270) X(288) X(320) X(324) X(336) X(360) X(378) X(384) X(400) X(416) X(432) X(448) X(480) X(486) X(504) X(512)

inline bool fft_length_supported(int n) {
  switch (n) {
    case 1:
#define EMC_CASE(L) case L:
    EMC_FOR_EACH_LENGTH(EMC_CASE)
#undef EMC_CASE
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

#ifdef __CUDACC__
// Asynchronous global -> shared copies of 8 bytes (cp.async, no register staging).  A thread's
// copies are complete after cp_async_wait<N>() leaves at most N of its committed groups pending;
// a barrier then publishes them to the other threads.
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Bulk global -> shared copies through the tensor-memory-access unit (cp.async.bulk, this CTA's
// own shared memory, no multicast), completed on a shared-memory mbarrier by transaction count.
// Source and destination 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(b), "r"(count) : "memory");
  // make the initialised barrier visible to the asynchronous proxy that completes it
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// Arrives on the barrier announcing `bytes` of transactions for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(b), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* smem_dst, const void* gmem_src, unsigned bytes, uint64_t* bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(d),
               "l"(gmem_src), "r"(bytes), "r"(b)
               : "memory");
}
// Orders this thread's earlier generic-proxy accesses to shared memory before later asynchronous-
// proxy ones (a bulk copy into a buffer the CTA has just read or written).
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// Waits for phase `parity` of the barrier to complete, giving up after about `max_cycles` SM
// clock cycles.  Returns whether it completed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long max_cycles) {
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(b), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > max_cycles) return false;
  }
}
#endif

}  // namespace emc
