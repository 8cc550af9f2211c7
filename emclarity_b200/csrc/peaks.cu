// peaks.cu -- template-search post-processing: greedy peak picking with rotated erase masks,
// and the local normalisation of the pre-processing.
//
// Peak picking (alignment/BH_templateSearch3d_2.m:1100-1275, nPeaks = 1): repeat
//   [MAX, coord] = max(mag(:))                    (first index among ties)
//   if Ang(coord) > 0: record samplingRate * (c + centre of mass of mag in the 3^3 box - rmDim),
//     ANGLE_LIST(Ang(coord), :) and MAX; rotate the removal mask by the peak's Euler angles
//     (interpolator 'forward', C1) and zero mag in the (2 rmDim + 1)^3 box where it is >= cutoff
//   else: mag(coord) = 0
// while n <= maxPeaks, tries < maxTries and MAX > highThr.
// B200 layout: the map stays in HBM; a per-tile (8^3) maximum key (ordered value << 32 | ~index,
// so ties keep the first index) is kept up to date, and each step reduces only the tile keys,
// then rewrites only the tiles the erase box touched.  Steps run in batches of device launches
// that stop by themselves once the loop condition fails (a device status word), so the host
// synchronises once per batch, not once per peak.
//
// Local normalisation (BH_templateSearch3d_2.m:558-561, statistics/BH_movingAverage_2.m):
// mean = Gaussian-weighted moving average (kernel length = feature size, sigma 3, centred on
// (L - 1) / 2, normalised; EMC_gaussianKernel + EMC_convn 'same' after symmetric padding by
// ceil(L / 2)), rms = sqrt(mean(x^2) - mean(x)^2), x <- (x - mean) / rms.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "interp.cuh"

namespace emc {
namespace {

constexpr int kTile = 8;

__device__ __forceinline__ unsigned long long peak_key(float v, unsigned lin) {
  const unsigned u = __float_as_uint(v);
  const unsigned k = (v != v) ? 0u : ((u & 0x80000000u) ? ~u : (u | 0x80000000u));  // NaN never wins
  return ((unsigned long long)k << 32) | (0xffffffffu - lin);
}
__device__ __forceinline__ float key_value(unsigned long long key) {
  const unsigned k = (unsigned)(key >> 32);
  const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}

struct PeakGeom {
  int nx, ny, nz;
  int tx, ty, tz;  // tiles per axis
  int rm;          // rmDim
  float cutoff;
  float sampling;
  float high_thr;
  int max_peaks, max_tries;
};

// Device state of the loop.
struct PeakState {
  int n_found;      // peaks recorded
  int tries;        // loop iterations
  int done;         // 1 once the loop condition failed
  int erase;        // 1: the last step recorded a peak and its box must be erased
  int cx, cy, cz;   // 0-based centre of the last step
  int angle;        // 1-based angle index of the last peak
  int reset_tile;   // tile to rescan after a single-voxel zeroing (-1 none)
  int pad;
};

// Maximum key of tile t.
__device__ unsigned long long tile_max(const float* mag, const PeakGeom& g, int t, int lane, int width) {
  const int tx = t % g.tx, ty = (t / g.tx) % g.ty, tz = t / (g.tx * g.ty);
  unsigned long long best = 0ull;
  for (int i = lane; i < kTile * kTile * kTile; i += width) {
    const int x = tx * kTile + (i & 7), y = ty * kTile + ((i >> 3) & 7), z = tz * kTile + (i >> 6);
    if (x < g.nx && y < g.ny && z < g.nz) {
      const unsigned lin = (unsigned)(((long)z * g.ny + y) * g.nx + x);
      const unsigned long long k = peak_key(mag[lin], lin);
      best = k > best ? k : best;
    }
  }
  return best;
}

__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// One warp per tile.
__global__ void k_tile_keys(const float* __restrict__ mag, PeakGeom g, unsigned long long* __restrict__ keys) {
  const int warps = blockDim.x >> 5;
  const long ntiles = (long)g.tx * g.ty * g.tz;
  for (long t = blockIdx.x * (long)warps + (threadIdx.x >> 5); t < ntiles; t += (long)gridDim.x * warps) {
    const unsigned long long k = warp_max(tile_max(mag, g, (int)t, threadIdx.x & 31, 32));
    if ((threadIdx.x & 31) == 0) keys[t] = k;
  }
}

// One step of the loop, one CTA: global max over the tile keys, the decision, the centre of mass
// and the record.
__global__ void __launch_bounds__(1024) k_peak_select(float* __restrict__ mag, const float* __restrict__ ang,
                                                      PeakGeom g, const unsigned long long* __restrict__ keys,
                                                      const double* __restrict__ angle_list, int n_angles,
                                                      PeakState* __restrict__ st, double* __restrict__ peaks) {
  __shared__ unsigned long long red[32];
  __shared__ int s_done;
  if (threadIdx.x == 0) s_done = st->done;
  __syncthreads();
  if (s_done) return;
  const long ntiles = (long)g.tx * g.ty * g.tz;
  unsigned long long best = 0ull;
  for (long t = threadIdx.x; t < ntiles; t += blockDim.x) best = keys[t] > best ? keys[t] : best;
  best = warp_max(best);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) best = red[w] > best ? red[w] : best;
  red[0] = best;
  PeakState s = *st;
  s.erase = 0;
  s.reset_tile = -1;
  const float mx = key_value(best);
  // while n <= maxPeaks && tries < maxTries && MAX > highThr
  if (!(s.n_found < g.max_peaks && s.tries < g.max_tries && best != 0ull && mx > g.high_thr)) {
    s.done = 1;
    *st = s;
    return;
  }
  s.tries += 1;
  const unsigned lin = 0xffffffffu - (unsigned)(best & 0xffffffffu);
  const int x = (int)(lin % (unsigned)g.nx), y = (int)((lin / (unsigned)g.nx) % (unsigned)g.ny),
            z = (int)(lin / ((unsigned)g.nx * (unsigned)g.ny));
  const float a = ang[lin];
  if (a > 0.f) {
    // centre of mass of mag in the 3^3 box around the peak (bDist = 1 + round(log(1)) = 1)
    double sw = 0.0, sx = 0.0, sy = 0.0, sz = 0.0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int xx = x + dx, yy = y + dy, zz = z + dz;
          if (xx < 0 || yy < 0 || zz < 0 || xx >= g.nx || yy >= g.ny || zz >= g.nz) continue;
          const double v = mag[((long)zz * g.ny + yy) * g.nx + xx];
          sw += v;
          sx += v * dx;
          sy += v * dy;
          sz += v * dz;
        }
    const int ai = (int)a;  // 1-based
    double* row = peaks + 10 * (size_t)s.n_found;
    // (c + cMass - rmDim) with c 1-based
    row[0] = g.sampling * ((x + 1) + sx / sw - g.rm);
    row[1] = g.sampling * ((y + 1) + sy / sw - g.rm);
    row[2] = g.sampling * ((z + 1) + sz / sw - g.rm);
    const bool in_list = ai >= 1 && ai <= n_angles;
    for (int k = 0; k < 3; ++k) row[3 + k] = in_list ? angle_list[3 * (size_t)(ai - 1) + k] : 0.0;
    row[6] = row[7] = row[8] = 0.0;
    row[9] = mx;
    s.n_found += 1;
    s.erase = 1;
    s.cx = x;
    s.cy = y;
    s.cz = z;
    s.angle = in_list ? ai : 0;
  } else {
    mag[lin] = 0.f;
    s.reset_tile = (z / kTile * g.ty + y / kTile) * g.tx + x / kTile;
  }
  *st = s;
}

// Zeroes mag in the (2 rm + 1)^3 box where the rotated removal mask is >= cutoff.  rmats: the
// sampling matrix (rows) of every angle, defineMatrix(angles, 'Bah', 'forward').
__global__ void k_peak_erase(float* __restrict__ mag, PeakGeom g, const PeakState* __restrict__ st,
                             const float* __restrict__ removal, const float* __restrict__ rmats) {
  const PeakState s = *st;
  if (!s.erase || s.done) return;
  const int r = 2 * g.rm + 1;
  const long nbox = (long)r * r * r;
  const float* m = rmats + 9 * (size_t)(s.angle > 0 ? s.angle - 1 : 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nbox; i += (long)gridDim.x * blockDim.x) {
    const int bx = (int)(i % r), by = (int)((i / r) % r), bz = (int)(i / ((long)r * r));
    const int x = s.cx - g.rm + bx, y = s.cy - g.rm + by, z = s.cz - g.rm + bz;
    if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) continue;
    // 'forward' with zero shift: s = R (p - c) + c, c = floor(r / 2) = rm, zero border
    const float u = (float)(bx - g.rm), v = (float)(by - g.rm), w = (float)(bz - g.rm);
    float rm_val = 1.f;  // no angle: erase the whole box
    if (s.angle > 0) {
      const float sx = fmaf(m[0], u, fmaf(m[1], v, m[2] * w)) + (float)g.rm;
      const float sy = fmaf(m[3], u, fmaf(m[4], v, m[5] * w)) + (float)g.rm;
      const float sz = fmaf(m[6], u, fmaf(m[7], v, m[8] * w)) + (float)g.rm;
      rm_val = sample_linear_border(removal, r, r, r, sx, sy, sz);
    }
    if (!(rm_val < g.cutoff)) mag[((long)z * g.ny + y) * g.nx + x] = 0.f;
  }
}

// Rescans the tiles the last step changed.
__global__ void k_peak_retile(const float* __restrict__ mag, PeakGeom g, const PeakState* __restrict__ st,
                              unsigned long long* __restrict__ keys) {
  const PeakState s = *st;
  const int warps = blockDim.x >> 5;
  const int wid = blockIdx.x * warps + (threadIdx.x >> 5);
  if (s.reset_tile >= 0) {
    if (wid == 0) {
      const unsigned long long k = warp_max(tile_max(mag, g, s.reset_tile, threadIdx.x & 31, 32));
      if ((threadIdx.x & 31) == 0) keys[s.reset_tile] = k;
    }
    return;
  }
  if (!s.erase) return;
  const int x0 = max(0, s.cx - g.rm) / kTile, x1 = min(g.nx - 1, s.cx + g.rm) / kTile;
  const int y0 = max(0, s.cy - g.rm) / kTile, y1 = min(g.ny - 1, s.cy + g.rm) / kTile;
  const int z0 = max(0, s.cz - g.rm) / kTile, z1 = min(g.nz - 1, s.cz + g.rm) / kTile;
  const int nx = x1 - x0 + 1, ny = y1 - y0 + 1, nt = nx * ny * (z1 - z0 + 1);
  for (int j = wid; j < nt; j += gridDim.x * warps) {
    const int t = ((z0 + j / (nx * ny)) * g.ty + (y0 + (j / nx) % ny)) * g.tx + (x0 + j % nx);
    const unsigned long long k = warp_max(tile_max(mag, g, t, threadIdx.x & 31, 32));
    if ((threadIdx.x & 31) == 0) keys[t] = k;
  }
}

// ---------------------------------------------------------------- moving average
// One separable pass along `axis` with symmetric (mirror, edge repeated) boundaries:
// out[x] = sum_t w[t] in[reflect(x + h - t)], h = floor(L / 2).
__global__ void k_mavg_pass(const float* __restrict__ in, float* __restrict__ out, int nx, int ny, int nz, int axis,
                            const float* __restrict__ w, int L) {
  const long n = (long)nx * ny * nz;
  const int h = L / 2;
  const int len = axis == 0 ? nx : axis == 1 ? ny : nz;
  const long stride = axis == 0 ? 1 : axis == 1 ? nx : (long)nx * ny;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const int pos = axis == 0 ? (int)(i % nx) : axis == 1 ? (int)((i / nx) % ny) : (int)(i / ((long)nx * ny));
    const long base = i - (long)pos * stride;
    float acc = 0.f;
    for (int t = 0; t < L; ++t) {
      int q = pos + h - t;
      // symmetric padding (padarray 'symmetric'): -1 -> 0, -2 -> 1, len -> len-1, ...
      if (q < 0) q = -q - 1;
      if (q >= len) q = 2 * len - q - 1;
      q = q < 0 ? 0 : (q >= len ? len - 1 : q);
      acc = fmaf(w[t], __ldg(in + base + (long)q * stride), acc);
    }
    out[i] = acc;
  }
}

__global__ void k_square(const float* __restrict__ in, float* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = in[i] * in[i];
}

__global__ void k_local_norm(float* __restrict__ x, const float* __restrict__ avg, const float* __restrict__ avg2,
                             long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float a = avg[i];
    const float rms = sqrtf(avg2[i] - a * a);
    x[i] = (x[i] - a) / rms;
  }
}

int grid1(long n) { return (int)std::max<long>(1, std::min<long>((n + 255) / 256, 8L * device_sm_count())); }

// The normalised kernel of EMC_gaussianKernel([1, L], 3) (masking/EMC_gaussianKernel.m), single precision,
// normalised again as BH_movingAverage_2 does.
std::vector<float> mavg_kernel(int L) {
  std::vector<float> w(L);
  float s = 0.f;
  for (int t = 0; t < L; ++t) {
    const float v = ((float)t - (float)(L - 1) / 2.f) / 3.f;
    w[t] = expf(-0.5f * v * v);
    s += w[t];
  }
  float s2 = 0.f;
  for (int t = 0; t < L; ++t) {
    w[t] /= s;
    s2 += w[t];
  }
  for (int t = 0; t < L; ++t) w[t] /= s2;
  return w;
}

emc_status mavg(const float* in, float* out, float* tmp, int nx, int ny, int nz, const float* d_w, int L,
                cudaStream_t st) {
  const long n = (long)nx * ny * nz;
  k_mavg_pass<<<grid1(n), 256, 0, st>>>(in, out, nx, ny, nz, 0, d_w, L);
  k_mavg_pass<<<grid1(n), 256, 0, st>>>(out, tmp, nx, ny, nz, 1, d_w, L);
  k_mavg_pass<<<grid1(n), 256, 0, st>>>(tmp, out, nx, ny, nz, 2, d_w, L);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

}  // namespace
}  // namespace emc

extern "C" {

emc_status emc_tsearch_peaks(float* d_mag, const float* d_ang, int nx, int ny, int nz, const float* h_removal,
                             int rm_dim, float mask_cutoff, const double* angle_list, int n_angles, int max_peaks,
                             int max_tries, float high_thr, float sampling, double* h_peaks, int* n_found,
                             void* stream) {
  EMC_CHECK_ARG(d_mag && d_ang && h_removal && angle_list && h_peaks && n_found, "emc_tsearch_peaks: null argument");
  EMC_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && (long)nx * ny * nz < 0xffffffffL, "emc_tsearch_peaks: bad size");
  EMC_CHECK_ARG(rm_dim >= 1 && rm_dim < 256, "emc_tsearch_peaks: rm_dim %d", rm_dim);
  EMC_CHECK_ARG(n_angles >= 1 && max_peaks >= 0 && max_tries >= 0, "emc_tsearch_peaks: bad counts");
  cudaStream_t st = emc::as_stream(stream);
  emc::PeakGeom g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.tx = (nx + emc::kTile - 1) / emc::kTile;
  g.ty = (ny + emc::kTile - 1) / emc::kTile;
  g.tz = (nz + emc::kTile - 1) / emc::kTile;
  g.rm = rm_dim;
  g.cutoff = mask_cutoff;
  g.sampling = sampling;
  g.high_thr = high_thr;
  g.max_peaks = max_peaks;
  g.max_tries = max_tries;
  const long ntiles = (long)g.tx * g.ty * g.tz;
  const int r = 2 * rm_dim + 1;
  // forward sampling matrices of every angle (rows), defineMatrix(angles, 'Bah', 'forward')
  std::vector<float> mats(9 * (size_t)n_angles);
  for (int a = 0; a < n_angles; ++a) {
    double R[9];
    EMC_TRY(emc_define_matrix(angle_list + 3 * (size_t)a, 0, R));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) mats[9 * (size_t)a + 3 * i + j] = (float)R[i + 3 * j];
  }
  unsigned long long* keys = nullptr;
  emc::PeakState* d_st = nullptr;
  float *d_rm = nullptr, *d_mats = nullptr;
  double *d_list = nullptr, *d_peaks = nullptr;
  emc_status rs = EMC_OK;
  auto alloc = [&](void** p, size_t b) {
    if (rs == EMC_OK && cudaMalloc(p, std::max<size_t>(b, 8)) != cudaSuccess) {
      emc::set_error("emc_tsearch_peaks: cudaMalloc(%zu) failed", b);
      rs = EMC_E_OOM;
    }
  };
  alloc((void**)&keys, sizeof(unsigned long long) * ntiles);
  alloc((void**)&d_st, sizeof(emc::PeakState));
  alloc((void**)&d_rm, sizeof(float) * (size_t)r * r * r);
  alloc((void**)&d_mats, sizeof(float) * mats.size());
  alloc((void**)&d_list, sizeof(double) * 3 * (size_t)n_angles);
  alloc((void**)&d_peaks, sizeof(double) * 10 * (size_t)std::max(1, max_peaks));
  emc::PeakState s0;
  memset(&s0, 0, sizeof(s0));
  s0.reset_tile = -1;
  if (rs == EMC_OK &&
      (cudaMemcpyAsync(d_st, &s0, sizeof(s0), cudaMemcpyHostToDevice, st) != cudaSuccess ||
       cudaMemcpyAsync(d_rm, h_removal, sizeof(float) * (size_t)r * r * r, cudaMemcpyHostToDevice, st) != cudaSuccess ||
       cudaMemcpyAsync(d_mats, mats.data(), sizeof(float) * mats.size(), cudaMemcpyHostToDevice, st) != cudaSuccess ||
       cudaMemcpyAsync(d_list, angle_list, sizeof(double) * 3 * (size_t)n_angles, cudaMemcpyHostToDevice, st) !=
           cudaSuccess))
    rs = EMC_E_CUDA;
  if (rs == EMC_OK) {
    emc::k_tile_keys<<<emc::grid1(ntiles * 32), 256, 0, st>>>(d_mag, g, keys);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  const int erase_blocks = (int)std::max<long>(1, std::min<long>(((long)r * r * r + 255) / 256, 256));
  emc::PeakState hs = s0;
  // batches of steps; each kernel returns at once after the loop condition failed
  constexpr int kBatch = 64;
  while (rs == EMC_OK && !hs.done) {
    for (int b = 0; b < kBatch && rs == EMC_OK; ++b) {
      emc::k_peak_select<<<1, 1024, 0, st>>>(d_mag, d_ang, g, keys, d_list, n_angles, d_st, d_peaks);
      emc::k_peak_erase<<<erase_blocks, 256, 0, st>>>(d_mag, g, d_st, d_rm, d_mats);
      emc::k_peak_retile<<<8, 256, 0, st>>>(d_mag, g, d_st, keys);
      if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
    }
    if (rs == EMC_OK && (cudaMemcpyAsync(&hs, d_st, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                         cudaStreamSynchronize(st) != cudaSuccess))
      rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK && hs.n_found > 0 &&
      (cudaMemcpyAsync(h_peaks, d_peaks, sizeof(double) * 10 * (size_t)hs.n_found, cudaMemcpyDeviceToHost, st) !=
           cudaSuccess ||
       cudaStreamSynchronize(st) != cudaSuccess))
    rs = EMC_E_CUDA;
  if (rs == EMC_E_CUDA) emc::set_error("emc_tsearch_peaks: %s", cudaGetErrorString(cudaGetLastError()));
  *n_found = rs == EMC_OK ? hs.n_found : 0;
  cudaStreamSynchronize(st);
  cudaFree(keys);
  cudaFree(d_st);
  cudaFree(d_rm);
  cudaFree(d_mats);
  cudaFree(d_list);
  cudaFree(d_peaks);
  return rs;
}

emc_status emc_moving_average(const float* d_in, int nx, int ny, int nz, int feature_size, float* d_out,
                              void* stream) {
  EMC_CHECK_ARG(d_in && d_out && nx > 0 && ny > 0 && nz > 0, "emc_moving_average: bad argument");
  EMC_CHECK_ARG(feature_size >= 2 && feature_size <= 2 * std::min(nx, std::min(ny, nz)),
                "emc_moving_average: feature size %d", feature_size);
  cudaStream_t st = emc::as_stream(stream);
  const std::vector<float> w = emc::mavg_kernel(feature_size);
  const long n = (long)nx * ny * nz;
  float *d_w = nullptr, *tmp = nullptr;
  EMC_CUDA(cudaMallocAsync((void**)&d_w, sizeof(float) * feature_size, st));
  emc_status rs = EMC_OK;
  if (cudaMallocAsync((void**)&tmp, sizeof(float) * n, st) != cudaSuccess) rs = EMC_E_OOM;
  if (rs == EMC_OK && cudaMemcpyAsync(d_w, w.data(), sizeof(float) * feature_size, cudaMemcpyHostToDevice, st) !=
                          cudaSuccess)
    rs = EMC_E_CUDA;
  if (rs == EMC_OK) rs = emc::mavg(d_in, d_out, tmp, nx, ny, nz, d_w, feature_size, st);
  if (rs == EMC_E_OOM) emc::set_error("emc_moving_average: scratch allocation failed");
  cudaStreamSynchronize(st);  // w (host) is read by the async copy
  cudaFreeAsync(tmp, st);
  cudaFreeAsync(d_w, st);
  return rs;
}

emc_status emc_local_normalize(float* d_vol, int nx, int ny, int nz, int feature_size, void* stream) {
  EMC_CHECK_ARG(d_vol && nx > 0 && ny > 0 && nz > 0, "emc_local_normalize: bad argument");
  EMC_CHECK_ARG(feature_size >= 2 && feature_size <= 2 * std::min(nx, std::min(ny, nz)),
                "emc_local_normalize: feature size %d", feature_size);
  cudaStream_t st = emc::as_stream(stream);
  const std::vector<float> w = emc::mavg_kernel(feature_size);
  const long n = (long)nx * ny * nz;
  float *d_w = nullptr, *buf = nullptr;
  EMC_CUDA(cudaMallocAsync((void**)&d_w, sizeof(float) * feature_size, st));
  emc_status rs = EMC_OK;
  if (cudaMallocAsync((void**)&buf, sizeof(float) * 4 * n, st) != cudaSuccess) rs = EMC_E_OOM;
  if (rs == EMC_OK && cudaMemcpyAsync(d_w, w.data(), sizeof(float) * feature_size, cudaMemcpyHostToDevice, st) !=
                          cudaSuccess)
    rs = EMC_E_CUDA;
  if (rs == EMC_OK) {
    float *avg = buf, *avg2 = buf + n, *sq = buf + 2 * n, *tmp = buf + 3 * n;
    rs = emc::mavg(d_vol, avg, tmp, nx, ny, nz, d_w, feature_size, st);
    if (rs == EMC_OK) {
      emc::k_square<<<emc::grid1(n), 256, 0, st>>>(d_vol, sq, n);
      rs = emc::mavg(sq, avg2, tmp, nx, ny, nz, d_w, feature_size, st);
    }
    if (rs == EMC_OK) {
      emc::k_local_norm<<<emc::grid1(n), 256, 0, st>>>(d_vol, avg, avg2, n);
      if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
    }
  }
  if (rs == EMC_E_OOM) emc::set_error("emc_local_normalize: scratch allocation failed");
  cudaStreamSynchronize(st);
  cudaFreeAsync(buf, st);
  cudaFreeAsync(d_w, st);
  return rs;
}

}  // extern "C"
