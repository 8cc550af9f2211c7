// fft_passes.cu -- launchers for the generic FFT passes and the mexFFT-style API.
#include <algorithm>
#include <atomic>
#include <new>

#include "fft_passes.cuh"

namespace emc {


static int grid_for(long work_items, int per_block) {
  long b = (work_items + per_block - 1) / per_block;
  long cap = 8L * device_sm_count();
  return (int)std::max(1L, std::min(b, cap));
}

template <int L>
static emc_status rows_r2c_t(const float* in, long in_pitch, float2* out, long out_pitch, long nrows,
                             cudaStream_t st) {
  constexpr int P = team_size(L);
  constexpr int TEAMS = rows_teams(L, P);
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  const long npairs = (nrows + 1) / 2;
  k_rows_r2c<L, P><<<grid_for(npairs, TEAMS), TEAMS * P, 0, st>>>(in, in_pitch, out, out_pitch, nrows, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

template <int L>
static emc_status rows_c2r_t(const float2* in, long in_pitch, float* out, long out_pitch, long nrows,
                             cudaStream_t st) {
  constexpr int P = team_size(L);
  constexpr int TEAMS = rows_teams(L, P);
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  const long npairs = (nrows + 1) / 2;
  k_rows_c2r<L, P><<<grid_for(npairs, TEAMS), TEAMS * P, 0, st>>>(in, in_pitch, out, out_pitch, nrows, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

template <int L, int SIGN>
static emc_status cols_t(const float2* in, float2* out, long stride, long inner, long outer, long outer_pitch,
                         cudaStream_t st) {
  using C = ColsCfg<L>;
  const float2* tw = device_twiddles(L);
  if (!tw) return EMC_E_CUDA;
  auto kern = k_cols<L, SIGN, C::P, C::T>;
  // CTAs per SM, per device: the first launch on a device queries it; threads that race there both
  // store the same value
  static std::atomic<int> resident[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64) return EMC_E_CUDA;
  int res = resident[dev].load(std::memory_order_acquire);
  if (!res) {
    if (C::smem > 48 * 1024)
      EMC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem));
    int nb = 0;
    EMC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, C::P * C::T, C::smem));
    res = std::max(nb, 1);
    resident[dev].store(res, std::memory_order_release);
  }
  const long units = (inner + C::T - 1) / C::T * outer;
  const long ctas = std::min<long>(units, (long)res * device_sm_count());
  kern<<<(unsigned)ctas, C::P * C::T, C::smem, st>>>(in, out, stride, inner, outer, outer_pitch, tw);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status launch_rows_r2c(int L, const float* in, long in_pitch, float2* out, long out_pitch, long nrows,
                           cudaStream_t st) {
  switch (L) {
#define X(n) case n: return rows_r2c_t<n>(in, in_pitch, out, out_pitch, nrows, st);
    EMC_FOR_EACH_LENGTH(X)
#undef X
    default: set_error("FFT length %d not supported", L); return EMC_E_UNSUPPORTED;
  }
}

emc_status launch_rows_c2r(int L, const float2* in, long in_pitch, float* out, long out_pitch, long nrows,
                           cudaStream_t st) {
  switch (L) {
#define X(n) case n: return rows_c2r_t<n>(in, in_pitch, out, out_pitch, nrows, st);
    EMC_FOR_EACH_LENGTH(X)
#undef X
    default: set_error("FFT length %d not supported", L); return EMC_E_UNSUPPORTED;
  }
}

emc_status launch_cols(int L, int sign, const float2* in, float2* out, long stride, long inner, long outer,
                       long outer_pitch, cudaStream_t st) {
  if (L == 1) {
    if (in != out) {
      set_error("launch_cols: L == 1 out of place not supported");
      return EMC_E_ARG;
    }
    return EMC_OK;
  }
  if (sign < 0) {
    switch (L) {
#define X(n) case n: return cols_t<n, -1>(in, out, stride, inner, outer, outer_pitch, st);
      EMC_FOR_EACH_LENGTH(X)
#undef X
    }
  } else {
    switch (L) {
#define X(n) case n: return cols_t<n, 1>(in, out, stride, inner, outer, outer_pitch, st);
      EMC_FOR_EACH_LENGTH(X)
#undef X
    }
  }
  set_error("FFT length %d not supported", L);
  return EMC_E_UNSUPPORTED;
}

emc_status fft3_r2c(const float* in, float2* out, int nx, int ny, int nz, int batch, cudaStream_t st) {
  const long nxh = nx / 2 + 1;
  const long rows = (long)ny * nz * batch;
  EMC_TRY(launch_rows_r2c(nx, in, nx, out, nxh, rows, st));
  if (ny > 1) EMC_TRY(launch_cols(ny, -1, out, out, nxh, nxh, (long)nz * batch, (long)ny * nxh, st));
  if (nz > 1) EMC_TRY(launch_cols(nz, -1, out, out, (long)ny * nxh, (long)ny * nxh, batch, (long)nz * ny * nxh, st));
  return EMC_OK;
}

emc_status fft3_c2r(const float2* in, float* out, float2* scratch, int nx, int ny, int nz, int batch,
                    cudaStream_t st) {
  const long nxh = nx / 2 + 1;
  const long rows = (long)ny * nz * batch;
  const float2* cur = in;
  if (nz > 1) {
    EMC_TRY(launch_cols(nz, 1, cur, scratch, (long)ny * nxh, (long)ny * nxh, batch, (long)nz * ny * nxh, st));
    cur = scratch;
  }
  if (ny > 1) {
    EMC_TRY(launch_cols(ny, 1, cur, scratch, nxh, nxh, (long)nz * batch, (long)ny * nxh, st));
    cur = scratch;
  }
  EMC_TRY(launch_rows_c2r(nx, cur, nxh, out, nx, rows, st));
  return EMC_OK;
}

}  // namespace emc

// ------------------------------------------------------------------ C-ABI: mexFFT
struct emc_fft_s {
  int dims[3];
  int batch;
  float2* scratch;
  size_t scratch_elems;
};

extern "C" {

emc_status emc_fft_plan(int rank, const int dims[3], int batch, emc_fft_t* out) {
  EMC_CHECK_ARG(out && dims, "emc_fft_plan: null argument");
  *out = nullptr;
  EMC_CHECK_ARG(rank >= 1 && rank <= 3, "emc_fft_plan: rank %d not in 1..3", rank);
  EMC_CHECK_ARG(batch >= 1, "emc_fft_plan: batch must be >= 1");
  int d[3] = {1, 1, 1};
  for (int i = 0; i < rank; ++i) d[i] = dims[i];
  EMC_CHECK_ARG(d[0] >= 2, "emc_fft_plan: nx must be >= 2");
  for (int i = 0; i < 3; ++i) {
    if (!emc::fft_length_supported(d[i])) {
      emc::set_error("emc_fft_plan: edge %d not a supported 2^a 3^b length <= 512", d[i]);
      return EMC_E_UNSUPPORTED;
    }
  }
  emc_fft_s* p = new (std::nothrow) emc_fft_s();
  EMC_CHECK_ARG(p, "emc_fft_plan: host allocation failed");
  for (int i = 0; i < 3; ++i) p->dims[i] = d[i];
  p->batch = batch;
  p->scratch_elems = (size_t)(d[0] / 2 + 1) * d[1] * d[2] * batch;
  p->scratch = nullptr;
  if (d[1] > 1 || d[2] > 1) {
    const size_t bytes = p->scratch_elems * sizeof(float2);
    cudaError_t e = cudaMalloc(&p->scratch, bytes);
    if (e != cudaSuccess) {
      delete p;
      emc::set_error("emc_fft_plan: cudaMalloc of %zu bytes failed", bytes);
      return EMC_E_OOM;
    }
  }
  // build the twiddle tables now so that later calls can be captured in a graph
  for (int i = 0; i < 3; ++i)
    if (d[i] > 1 && !emc::device_twiddles(d[i])) {
      cudaFree(p->scratch);
      delete p;
      return EMC_E_CUDA;
    }
  *out = p;
  return EMC_OK;
}

emc_status emc_fft_r2c(emc_fft_t p, const float* d_in, float* d_out, void* stream) {
  EMC_CHECK_ARG(p && d_in && d_out, "emc_fft_r2c: null argument");
  return emc::fft3_r2c(d_in, reinterpret_cast<float2*>(d_out), p->dims[0], p->dims[1], p->dims[2], p->batch,
                       emc::as_stream(stream));
}

emc_status emc_fft_c2r(emc_fft_t p, const float* d_in, float* d_out, void* stream) {
  EMC_CHECK_ARG(p && d_in && d_out, "emc_fft_c2r: null argument");
  return emc::fft3_c2r(reinterpret_cast<const float2*>(d_in), d_out, p->scratch, p->dims[0], p->dims[1],
                       p->dims[2], p->batch, emc::as_stream(stream));
}

emc_status emc_fft_destroy(emc_fft_t p) {
  if (!p) return EMC_OK;
  if (p->scratch) cudaFree(p->scratch);
  delete p;
  return EMC_OK;
}

}  // extern "C"
