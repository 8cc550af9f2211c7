// common.cu -- error text, twiddle tables, version string.
#include <math.h>
#include <stdarg.h>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace emc {

static thread_local char g_last_error[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

namespace {
constexpr int kMaxDevices = 64;
#define EMC_LEN_ITEM(L) L,
constexpr int kLengths[] = {EMC_FOR_EACH_LENGTH(EMC_LEN_ITEM)};
#undef EMC_LEN_ITEM
constexpr int kNumLengths = sizeof(kLengths) / sizeof(kLengths[0]);

struct DeviceTables {
  float2* base = nullptr;
  int offset[kNumLengths] = {0};
  bool ready = false;
};
DeviceTables g_tables[kMaxDevices];
std::mutex g_tables_mutex;
int g_sm_count[kMaxDevices] = {0};
}  // namespace

const float2* device_twiddles(int L) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error("device_twiddles: no current CUDA device");
    return nullptr;
  }
  int li = -1;
  for (int i = 0; i < kNumLengths; ++i)
    if (kLengths[i] == L) li = i;
  if (li < 0) {
    set_error("device_twiddles: FFT length %d not supported", L);
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_tables_mutex);
  DeviceTables& t = g_tables[dev];
  if (!t.ready) {
    std::vector<float2> host;
    for (int i = 0; i < kNumLengths; ++i) {
      t.offset[i] = (int)host.size();
      const int n = kLengths[i];
      for (int m = 0; m < n; ++m) {
        // exp(-2 pi i m / n) evaluated in double precision
        const double a = -2.0 * M_PI * (double)m / (double)n;
        host.push_back(make_float2((float)cos(a), (float)sin(a)));
      }
      // pad each table to a multiple of 4 entries (32-byte alignment)
      while (host.size() % 4) host.push_back(make_float2(0.f, 0.f));
    }
    float2* d = nullptr;
    if (cudaMalloc(&d, host.size() * sizeof(float2)) != cudaSuccess) {
      set_error("device_twiddles: cudaMalloc failed");
      return nullptr;
    }
    if (cudaMemcpy(d, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaFree(d);
      set_error("device_twiddles: cudaMemcpy failed");
      return nullptr;
    }
    t.base = d;
    t.ready = true;
  }
  return t.base + t.offset[li];
}

int device_sm_count() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  if (g_sm_count[dev] == 0) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    g_sm_count[dev] = n > 0 ? n : 148;
  }
  return g_sm_count[dev];
}

}  // namespace emc

extern "C" {

const char* emc_status_string(emc_status s) {
  switch (s) {
    case EMC_OK: return "ok";
    case EMC_E_ARG: return "invalid argument";
    case EMC_E_CUDA: return "CUDA error";
    case EMC_E_OOM: return "out of device memory";
    case EMC_E_TIMEOUT: return "device-side wait timed out";
    case EMC_E_UNSUPPORTED: return "unsupported size or mode";
    default: return "unknown status";
  }
}

const char* emc_last_error(void) { return emc::g_last_error; }

const char* emc_version(void) { return "emclarity_b200 0.1 (sm_100a)"; }

}  // extern "C"
