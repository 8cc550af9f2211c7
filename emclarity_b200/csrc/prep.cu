// prep.cu -- the volume / spectrum operators around the search:
//   emc_pad3d              BH_padZeros3d (masking/BH_padZeros3d.m:79-229): trim / pad with a fill
//                          value, optional 7-voxel cosine edge taper ('singleTaper')
//   emc_bandpass3d         BH_bandpass3d (masking/BH_bandpass3d.m:54-170) on the half spectrum
//   emc_band_limit_center_normalize
//                          BH_bandLimitCenterNormalize (masking/BH_bandLimitCenterNormalize.m:40-61)
//   emc_xcf_rotational     BH_multi_xcf_Rotational (statistics/BH_multi_xcf_Rotational.m:71-78)
//   emc_xcf_translational  BH_multi_xcf_Translational (statistics/BH_multi_xcf_Translational.m:31-104)
#include <math.h>

#include <algorithm>
#include <vector>

#include "fft_passes.cuh"

namespace emc {

// taper = 0.5 + 0.5 cos(((1:7)-1) pi / 7) (BH_padZeros3d.m:111-117); index i counts from the edge.
__device__ __forceinline__ float edge_taper(int i, int n) {
  float t = 1.f;
  if (i < 7) t *= 0.5f + 0.5f * cospif((float)(6 - i) / 7.0f);
  if (n - 1 - i < 7) t *= 0.5f + 0.5f * cospif((float)(6 - (n - 1 - i)) / 7.0f);
  return t;
}

struct PadGeom {
  int ix, iy, iz;        // input size
  int tx, ty, tz;        // trimmed size
  int tlx, tly, tlz;     // trim low
  int plx, ply, plz;     // pad low
  int ox, oy, oz;        // output size
  float fill;
  int taper;
};

__global__ void k_pad3d(const float* __restrict__ in, const PadGeom g, float* __restrict__ out) {
  const long total = (long)g.ox * g.oy * g.oz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.ox), y = (int)((i / g.ox) % g.oy), z = (int)(i / ((long)g.ox * g.oy));
    const int ax = x - g.plx, ay = y - g.ply, az = z - g.plz;
    float v = g.fill;
    if (ax >= 0 && ay >= 0 && az >= 0 && ax < g.tx && ay < g.ty && az < g.tz) {
      v = in[((long)(az + g.tlz) * g.iy + (ay + g.tly)) * g.ix + (ax + g.tlx)];
      if (g.taper) {
        const float t = edge_taper(ax, g.tx) * edge_taper(ay, g.ty) * edge_taper(az, g.tz);
        v = v * t + g.fill * (1.f - t);
      }
    }
    out[i] = v;
  }
}

// Bandpass window on the half spectrum, FFT order, radius in cycles / pixel.
__global__ void k_bandpass(int nx, int ny, int nz, float low_cut, float low_roll, float high_cut, float high_roll,
                           float* __restrict__ out) {
  const int nxh = nx / 2 + 1;
  const long total = (long)nxh * ny * nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nxh), y0 = (int)((i / nxh) % ny), z0 = (int)(i / ((long)nxh * ny));
    const int y = y0 <= ny / 2 ? y0 : y0 - ny, z = z0 <= nz / 2 ? z0 : z0 - nz;
    const float fx = (float)x / nx, fy = (float)y / ny, fz = nz > 1 ? (float)z / nz : 0.f;
    const float r = sqrtf(fx * fx + fy * fy + fz * fz);
    float w = r < low_cut ? 1.f : expf(-(r - low_cut) * (r - low_cut) / (2.f * low_roll * low_roll));
    if (high_cut != 0.f && r <= high_cut) w = expf(-(r - high_cut) * (r - high_cut) / (2.f * high_roll * high_roll));
    out[i] = w;
  }
}

template <typename Tv>
__device__ __forceinline__ void block_add(Tv v, Tv* red, Tv* target) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    Tv t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(target, t);
  }
}

__global__ void k_sum(const float* __restrict__ v, long n, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += v[i];
  block_add(s, red, out);
}

// F(0) = 0, F *= bandpass, accumulate sum_full |F|^2 (BH_bandLimitCenterNormalize.m:51-61)
__global__ void k_center_band(float2* __restrict__ f, const float* __restrict__ bp, long nhalf, int nxh, int nx,
                              double* __restrict__ energy) {
  __shared__ double red[32];
  double e = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nhalf; i += (long)gridDim.x * blockDim.x) {
    float2 v = f[i];
    float w = bp ? bp[i] : 1.f;
    if (i == 0) w = 0.f;
    v.x *= w;
    v.y *= w;
    f[i] = v;
    const int kx = (int)(i % nxh);
    e += (kx == 0 || 2 * kx == nx ? 1.0 : 2.0) * ((double)v.x * v.x + (double)v.y * v.y);
  }
  block_add(e, red, energy);
}

__global__ void k_scale_c(float2* __restrict__ f, long n, const double* __restrict__ energy, double numel) {
  const float s = (float)(numel / sqrt(*energy));
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    f[i].x *= s;
    f[i].y *= s;
  }
}

// numerator / denominators of BH_multi_xcf_Rotational.m:73-78 over the half spectrum (Hermitian weights)
__global__ void k_xcf_rot(const float2* __restrict__ p, const float2* __restrict__ r, const float* __restrict__ wa,
                          const float* __restrict__ wb, long nhalf, int nxh, int nx, double* __restrict__ sums) {
  __shared__ double red[3][32];
  double a = 0, b = 0, c = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nhalf; i += (long)gridDim.x * blockDim.x) {
    const int kx = (int)(i % nxh);
    const double h = (kx == 0 || 2 * kx == nx) ? 1.0 : 2.0;
    const float fa = wa ? wa[i] : 1.f, fb = wb ? wb[i] : 1.f;
    const float2 pv = p[i], rv = r[i];
    // refWdg .* P .* R .* wdgMask  (R is the conjugated reference spectrum)
    a += h * (double)fa * fb * ((double)pv.x * rv.x - (double)pv.y * rv.y);
    b += h * (double)fb * fb * ((double)rv.x * rv.x + (double)rv.y * rv.y);
    c += h * (double)fa * fa * ((double)pv.x * pv.x + (double)pv.y * pv.y);
  }
  double v[3] = {a, b, c};
  for (int k = 0; k < 3; ++k) {
    double t = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = t;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    atomicAdd(sums + threadIdx.x, t);
  }
}

__global__ void k_mul_c(const float2* __restrict__ a, const float2* __restrict__ b, float2* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = cmul(a[i], b[i]);
}

// min over the (unshifted) map; masked argmax in fftshifted column-major order, first index wins
__global__ void k_map_min(const float* __restrict__ m, long n, unsigned int* __restrict__ kmin) {
  unsigned int best = 0xffffffffu;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    best = min(best, ordered_key(m[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMin(kmin, best);
}

__global__ void k_map_argmax(const float* __restrict__ m, int nx, int ny, int nz, const float* __restrict__ pmask,
                             const unsigned int* __restrict__ kmin, unsigned long long* __restrict__ best) {
  const long n = (long)nx * ny * nz;
  const float minv = key_to_float(*kmin);
  unsigned long long b = 0ull;
  for (long s = blockIdx.x * (long)blockDim.x + threadIdx.x; s < n; s += (long)gridDim.x * blockDim.x) {
    // s: fftshifted index; unshifted source index
    const int xs = (int)(s % nx), ys = (int)((s / nx) % ny), zs = (int)(s / ((long)nx * ny));
    const int xu = (xs + nx - nx / 2) % nx, yu = (ys + ny - ny / 2) % ny, zu = (zs + nz - nz / 2) % nz;
    float v = m[((long)zu * ny + yu) * nx + xu];
    if (pmask && pmask[s] < 0.95f) v = minv;
    if (v != v) continue;
    const unsigned long long k = ((unsigned long long)ordered_key(v) << 32) | (0xffffffffu - (unsigned int)s);
    b = k > b ? k : b;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, b, o);
    b = t > b ? t : b;
  }
  if ((threadIdx.x & 31) == 0 && b) atomicMax(best, b);
}

}  // namespace emc

extern "C" {

emc_status emc_pad3d(const float* d_in, int nx, int ny, int nz, const int pad_low[3], const int pad_top[3],
                     float fill, int taper, float* d_out, void* stream) {
  EMC_CHECK_ARG(d_in && d_out && pad_low && pad_top, "emc_pad3d: null argument");
  emc::PadGeom g;
  g.ix = nx; g.iy = ny; g.iz = nz;
  const int in_d[3] = {nx, ny, nz};
  int tl[3], pl[3], td[3], od[3];
  for (int a = 0; a < 3; ++a) {
    tl[a] = pad_low[a] < 0 ? -pad_low[a] : 0;
    const int tt = pad_top[a] < 0 ? -pad_top[a] : 0;
    pl[a] = pad_low[a] > 0 ? pad_low[a] : 0;
    const int pt = pad_top[a] > 0 ? pad_top[a] : 0;
    td[a] = in_d[a] - tl[a] - tt;
    EMC_CHECK_ARG(td[a] > 0, "emc_pad3d: trimming removes the whole axis %d", a);
    od[a] = td[a] + pl[a] + pt;
  }
  g.tx = td[0]; g.ty = td[1]; g.tz = td[2];
  g.tlx = tl[0]; g.tly = tl[1]; g.tlz = tl[2];
  g.plx = pl[0]; g.ply = pl[1]; g.plz = pl[2];
  g.ox = od[0]; g.oy = od[1]; g.oz = od[2];
  g.fill = fill;
  g.taper = taper;
  const long total = (long)od[0] * od[1] * od[2];
  const int blocks = (int)std::min<long>((total + 255) / 256, 4L * emc::device_sm_count());
  emc::k_pad3d<<<std::max(blocks, 1), 256, 0, emc::as_stream(stream)>>>(d_in, g, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_bandpass3d(int nx, int ny, int nz, float high_thresh, float high_cut, float low_cut, float pixel_size,
                          float* d_out, void* stream) {
  EMC_CHECK_ARG(d_out && nx > 0 && ny > 0 && nz > 0, "emc_bandpass3d: bad argument");
  float lc, lr, hc = 0.f, hr = 0.f;
  const int mn = nz > 1 ? std::min(nx, std::min(ny, nz)) : std::min(nx, ny);
  if (pixel_size > 0.f) {
    // calc_frequencies (BH_bandpass3d.m:100-160)
    EMC_CHECK_ARG(high_thresh >= 0.f && high_thresh < 1.f, "emc_bandpass3d: HIGH_THRESH must be in [0, 1)");
    EMC_CHECK_ARG(low_cut != 0.f, "emc_bandpass3d: LOW_CUT must be non-zero");
    if (high_cut != 0.f) hc = pixel_size / high_cut;
    lc = pixel_size / low_cut;
    if (lc > 0.f) {
      lr = 2.0f / (float)mn;
    } else {
      lc = fabsf(lc);
      const float low_end = 0.5f;
      lr = sqrtf(-(low_end - lc) * (low_end - lc) / (2.f * logf(1e-3f)));
    }
    if (high_cut != 0.f) hr = sqrtf(-hc * hc / (2.f * logf(high_thresh)));
  } else {
    // 'nyquist' (pixel_size == 0) or 'nyquistHigh' (pixel_size < 0) (BH_bandpass3d.m:60-77)
    if (pixel_size < 0.f) {
      hc = 7.0f / (float)mn;
      hr = sqrtf(-hc * hc / (2.f * logf(1e-6f)));
    }
    lr = 1.5f / (float)mn;
    lc = 0.485f + low_cut;
  }
  const long total = (long)(nx / 2 + 1) * ny * nz;
  const int blocks = (int)std::min<long>((total + 255) / 256, 4L * emc::device_sm_count());
  emc::k_bandpass<<<std::max(blocks, 1), 256, 0, emc::as_stream(stream)>>>(nx, ny, nz, lc, lr, hc, hr, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_band_limit_center_normalize(const float* d_img, int nx, int ny, int nz, const int pad_low[3],
                                           const int pad_top[3], int taper, const float* d_bandpass,
                                           float* d_spectrum_out, void* stream) {
  EMC_CHECK_ARG(d_img && d_spectrum_out && pad_low && pad_top, "emc_band_limit_center_normalize: null argument");
  cudaStream_t st = emc::as_stream(stream);
  int od[3];
  const int in_d[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) od[a] = in_d[a] + pad_low[a] + pad_top[a];
  for (int a = 0; a < 3; ++a)
    EMC_CHECK_ARG(emc::fft_length_supported(od[a]) && od[a] >= 2, "padded edge %d not a supported FFT length", od[a]);
  const long nin = (long)nx * ny * nz, nout = (long)od[0] * od[1] * od[2];
  const long nhalf = (long)(od[0] / 2 + 1) * od[1] * od[2];
  char* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, sizeof(float) * nout + 64, st));
  double* sums = reinterpret_cast<double*>(buf);
  float* padded = reinterpret_cast<float*>(buf + 64);
  emc_status rs = EMC_OK;
  double mean = 0.0;
  // mean of the image (padding value, BH_bandLimitCenterNormalize.m:48)
  if (cudaMemsetAsync(sums, 0, 2 * sizeof(double), st) != cudaSuccess) rs = EMC_E_CUDA;
  if (rs == EMC_OK) {
    emc::k_sum<<<std::min<long>((nin + 255) / 256, 2L * emc::device_sm_count()), 256, 0, st>>>(d_img, nin, sums);
    if (cudaMemcpyAsync(&mean, sums, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK) rs = emc_pad3d(d_img, nx, ny, nz, pad_low, pad_top, (float)(mean / nin), taper, padded, stream);
  float2* f = reinterpret_cast<float2*>(d_spectrum_out);
  if (rs == EMC_OK) rs = emc::fft3_r2c(padded, f, od[0], od[1], od[2], 1, st);
  if (rs == EMC_OK) {
    const int blocks = (int)std::min<long>((nhalf + 255) / 256, 2L * emc::device_sm_count());
    emc::k_center_band<<<blocks, 256, 0, st>>>(f, d_bandpass, nhalf, od[0] / 2 + 1, od[0], sums + 1);
    emc::k_scale_c<<<blocks, 256, 0, st>>>(f, nhalf, sums + 1, (double)nout);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  cudaFreeAsync(buf, st);
  if (rs == EMC_E_CUDA) emc::set_error("emc_band_limit_center_normalize: CUDA failure");
  return rs;
}

emc_status emc_xcf_rotational(const float* d_part_ft, const float* d_ref_ft_conj, const float* d_wdg_mask,
                              const float* d_ref_wdg, int nx, int ny, int nz, double* h_cc, void* stream) {
  EMC_CHECK_ARG(d_part_ft && d_ref_ft_conj && h_cc, "emc_xcf_rotational: null argument");
  cudaStream_t st = emc::as_stream(stream);
  double* d = nullptr;
  EMC_CUDA(cudaMallocAsync(&d, 3 * sizeof(double), st));
  double h[3] = {0, 0, 0};
  emc_status rs = EMC_OK;
  const long nhalf = (long)(nx / 2 + 1) * ny * nz;
  if (cudaMemsetAsync(d, 0, 3 * sizeof(double), st) != cudaSuccess) rs = EMC_E_CUDA;
  if (rs == EMC_OK) {
    // wdgMask multiplies the (conjugated) reference, refWdg the particle
    emc::k_xcf_rot<<<std::min<long>((nhalf + 255) / 256, 2L * emc::device_sm_count()), 256, 0, st>>>(
        reinterpret_cast<const float2*>(d_part_ft), reinterpret_cast<const float2*>(d_ref_ft_conj), d_ref_wdg,
        d_wdg_mask, nhalf, nx / 2 + 1, nx, d);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rs = EMC_E_CUDA;
  }
  cudaFreeAsync(d, st);
  if (rs != EMC_OK) {
    emc::set_error("emc_xcf_rotational: CUDA failure");
    return rs;
  }
  *h_cc = h[0] / sqrt(h[1] * h[2]);
  return EMC_OK;
}

emc_status emc_xcf_translational(const float* d_a, const float* d_b, int nx, int ny, int nz, const float* d_peak_mask,
                                 int peak_com, double peak_out[3], double* max_val, float* d_map_out, void* stream) {
  EMC_CHECK_ARG(d_a && d_b && peak_out, "emc_xcf_translational: null argument");
  EMC_CHECK_ARG(peak_com >= 0 && peak_com < 32, "emc_xcf_translational: peak_com %d", peak_com);
  cudaStream_t st = emc::as_stream(stream);
  const long nhalf = (long)(nx / 2 + 1) * ny * nz, nvox = (long)nx * ny * nz;
  char* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, sizeof(float2) * 2 * nhalf + sizeof(float) * nvox + 64, st));
  unsigned long long* d_best = reinterpret_cast<unsigned long long*>(buf);
  unsigned int* d_kmin = reinterpret_cast<unsigned int*>(buf + 8);
  float2* prod = reinterpret_cast<float2*>(buf + 64);
  float2* scratch = prod + nhalf;
  float* map = reinterpret_cast<float*>(scratch + nhalf);
  emc_status rs = EMC_OK;
  const int blocks = (int)std::min<long>((nvox + 255) / 256, 4L * emc::device_sm_count());
  emc::k_mul_c<<<blocks, 256, 0, st>>>(reinterpret_cast<const float2*>(d_a), reinterpret_cast<const float2*>(d_b),
                                       prod, nhalf);
  if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  if (rs == EMC_OK) rs = emc::fft3_c2r(prod, map, scratch, nx, ny, nz, 1, st);
  unsigned long long best = 0;
  unsigned int kmin = 0;
  std::vector<float> hmap, hmask;
  if (rs == EMC_OK && d_peak_mask) {
    hmask.resize(nvox);
    if (cudaMemcpyAsync(hmask.data(), d_peak_mask, sizeof(float) * nvox, cudaMemcpyDeviceToHost, st)) rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK) {
    cudaMemsetAsync(d_best, 0, 8, st);
    cudaMemsetAsync(d_kmin, 0xff, 4, st);
    emc::k_map_min<<<blocks, 256, 0, st>>>(map, nvox, d_kmin);
    emc::k_map_argmax<<<blocks, 256, 0, st>>>(map, nx, ny, nz, d_peak_mask, d_kmin, d_best);
    hmap.resize(nvox);
    if (cudaGetLastError() != cudaSuccess || cudaMemcpyAsync(&best, d_best, 8, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(&kmin, d_kmin, 4, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(hmap.data(), map, sizeof(float) * nvox, cudaMemcpyDeviceToHost, st) ||
        cudaStreamSynchronize(st))
      rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK && d_map_out) {
    // fftshifted copy of the map, scaled by 1/numel like MATLAB ifftn
    std::vector<float> shifted(nvox);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
          shifted[((long)((z + nz / 2) % nz) * ny + (y + ny / 2) % ny) * nx + (x + nx / 2) % nx] =
              hmap[((long)z * ny + y) * nx + x] / (float)nvox;
    if (cudaMemcpyAsync(d_map_out, shifted.data(), sizeof(float) * nvox, cudaMemcpyHostToDevice, st) ||
        cudaStreamSynchronize(st))
      rs = EMC_E_CUDA;
  }
  cudaFreeAsync(buf, st);
  if (rs != EMC_OK) {
    emc::set_error("emc_xcf_translational: CUDA failure");
    return rs;
  }
  const int c[3] = {nx / 2, ny / 2, nz / 2};
  const int dims[3] = {nx, ny, nz};
  if (best == 0) {
    peak_out[0] = peak_out[1] = peak_out[2] = 0;
    if (max_val) *max_val = NAN;
    return EMC_OK;
  }
  const float minv = emc::key_to_float(kmin);
  const unsigned int s = 0xffffffffu - (unsigned int)(best & 0xffffffffull);
  const float mv = emc::key_to_float((unsigned int)(best >> 32));
  if (max_val) *max_val = mv / (double)nvox;
  double pc[3] = {(double)(s % nx), (double)((s / nx) % ny), (double)(s / ((long)nx * ny))};
  // two centre-of-mass passes on the (2k+1)^3 box of map - min (BH_multi_xcf_Translational.m:47-91)
  // value of the masked, fftshifted map (peakMask < 0.95 -> min, :33-34)
  auto at = [&](int xs, int ys, int zs) -> double {
    if (!hmask.empty() && hmask[((long)zs * ny + ys) * nx + xs] < 0.95f) return minv;
    const int xu = (xs + nx - c[0]) % nx, yu = (ys + ny - c[1]) % ny, zu = (zs + nz - c[2]) % nz;
    return hmap[((long)zu * ny + yu) * nx + xu];
  };
  if (mv != 0.f && peak_com > 0) {
    for (int it = 0; it < 2; ++it) {
      double base[3];
      for (int a = 0; a < 3; ++a) base[a] = it == 1 ? floor(pc[a] + 0.5) : pc[a];
      double sum = 0, cm[3] = {0, 0, 0};
      for (int dz = -peak_com; dz <= peak_com; ++dz)
        for (int dy = -peak_com; dy <= peak_com; ++dy)
          for (int dx = -peak_com; dx <= peak_com; ++dx) {
            const int p[3] = {(int)base[0] + dx, (int)base[1] + dy, (int)base[2] + dz};
            if (p[0] < 0 || p[1] < 0 || p[2] < 0 || p[0] >= dims[0] || p[1] >= dims[1] || p[2] >= dims[2]) {
              emc::set_error("emc_xcf_translational: centre-of-mass box leaves the map");
              return EMC_E_ARG;
            }
            const double v = at(p[0], p[1], p[2]) - minv;
            sum += v; cm[0] += v * dx; cm[1] += v * dy; cm[2] += v * dz;
          }
      for (int a = 0; a < 3; ++a) pc[a] = base[a] + cm[a] / sum;
    }
  }
  for (int a = 0; a < 3; ++a) peak_out[a] = pc[a] - c[a];
  for (int a = 0; a < 3; ++a)
    if (peak_out[a] != peak_out[a]) peak_out[a] = 0;
  return EMC_OK;
}

}  // extern "C"
