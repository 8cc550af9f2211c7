// masks.cu -- the weights and masks built once per reference or tilt range around the search:
//   emc_binary_wedge   BH_weightMask3d(.., 'binaryWedgeGPU') (masking/BH_weightMask3d.m:99-143)
//   emc_mask_sphere    EMC_maskShape('sphere', SIZE, RADIUS, ..) (masking/EMC_maskShape.m:95-224)
//   emc_cref_filter    BH_multi_cRef(fscINFO, radialGrid, ..) (statistics/BH_multi_cRef.m:1-166)
// Each is a handful of elementwise / separable-convolution launches over one volume; scratch is
// taken from the stream-ordered allocator and returned before the call ends.
#include <math.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace emc {
namespace {

constexpr int kMaxTaps = 63;
struct Taps {
  float w[kMaxTaps];
  int len;
};

// 'same' convolution with zero padding along one axis (convn(.., 'same') with a symmetric kernel,
// which equals the correlation written here).
__global__ void k_conv_axis(const float* __restrict__ in, float* __restrict__ out, int nx, int ny, int nz, int axis,
                            const Taps t) {
  const long total = (long)nx * ny * nz;
  const int h = (t.len - 1) / 2;
  const long stride = axis == 0 ? 1 : (axis == 1 ? (long)nx : (long)nx * ny);
  const int extent = axis == 0 ? nx : (axis == 1 ? ny : nz);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int p = axis == 0 ? (int)(i % nx) : (axis == 1 ? (int)((i / nx) % ny) : (int)(i / ((long)nx * ny)));
    float acc = 0.f;
    for (int k = 0; k < t.len; ++k) {
      const int q = p + k - h;
      if (q >= 0 && q < extent) acc = fmaf(t.w[k], __ldg(in + i + (long)(k - h) * stride), acc);
    }
    out[i] = acc;
  }
}

// keys[0] = ordered key of the minimum, keys[1] = of the maximum (finite values)
__global__ void k_minmax(const float* __restrict__ v, long n, unsigned* __restrict__ keys) {
  unsigned lo = 0xffffffffu, hi = 0u;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const unsigned k = ordered_key(v[i]);
    lo = min(lo, k);
    hi = max(hi, k);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(keys, lo);
    atomicMax(keys + 1, hi);
  }
}

// BH_bandpass3d(SIZE, 0, 0, 0, METHOD, 'nyquist') at centred coordinates (X, Y, Z): 1 below 0.485
// cycles per pixel, a Gaussian roll-off of width 1.5 / n beyond (masking/BH_bandpass3d.m:60-77)
__device__ __forceinline__ float nyquist_window(int X, int Y, int Z, int n) {
  const float rn = sqrtf((float)(X * X + Y * Y + Z * Z)) / (float)n;
  if (rn < 0.485f) return 1.f;
  const float roll = 1.5f / (float)n;
  return expf(-(rn - 0.485f) * (rn - 0.485f) / (2.f * roll * roll));
}

// Binary wedge on the centred n^3 grid (BH_weightMask3d.m:108-120): theta = atand2(X, Z); the cones
// (180 - minTilt <= theta | theta <= maxTilt - 180) | (-minTilt <= theta <= maxTilt) are removed and
// the |X|, |Z| <= 2 slab through the origin is kept.
__global__ void k_wedge_binary(int n, double max_cone, double min_cone, float* __restrict__ out) {
  const long total = (long)n * n * n;
  const int c = n / 2;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int X = (int)(i % n) - c, Z = (int)(i / ((long)n * n)) - c;
    const double theta = atan2((double)X, (double)Z) * (180.0 / 3.14159265358979323846);
    const bool excluded = (180.0 - min_cone <= theta || theta <= max_cone - 180.0) ||
                          (-min_cone <= theta && theta <= max_cone);
    float w = excluded ? 0.f : 1.f;
    if (abs(X) <= 2 && abs(Z) <= 2) w = 1.f;
    out[i] = w;
  }
}

__global__ void k_times_nyquist(float* __restrict__ v, int n) {
  const long total = (long)n * n * n;
  const int c = n / 2;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int X = (int)(i % n) - c, Y = (int)((i / n) % n) - c, Z = (int)(i / ((long)n * n)) - c;
    v[i] *= nyquist_window(X, Y, Z, n);
  }
}

// (W - min) / max(W - min), written centred (layout 0) or as the ifftshifted half spectrum in FFT
// order (layout 1: element (p, q, r), p <= n/2, reads centred index ((p + c) % n, ...)).
__global__ void k_wedge_normalise(const float* __restrict__ w, int n, const unsigned* __restrict__ keys, int layout,
                                  float* __restrict__ out) {
  const float lo = key_to_float(keys[0]);
  const float span = key_to_float(keys[1]) - lo;
  const int nh = n / 2 + 1, c = n / 2;
  const long total = layout ? (long)nh * n * n : (long)n * n * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    long src = i;
    if (layout) {
      const int p = (int)(i % nh), q = (int)((i / nh) % n), r = (int)(i / ((long)nh * n));
      src = ((long)((r + c) % n) * n + (q + c) % n) * n + (p + c) % n;
    }
    out[i] = (w[src] - lo) / span;
  }
}

// Binary ellipsoid of EMC_maskShape('sphere') with its zero taper: coordinates i - floor(n/2) - shift
// (EMC_coordVectors, origin 1), ((X/Rx)^2 + (Y/Ry)^2) + (Z/Rz)^2 <= 1 evaluated in single precision as
// MATLAB does, and the outer `taper` slices of every face set to 0 (EMC_resize 'force_taper' with a
// zero taper).
__global__ void k_sphere_binary(int nx, int ny, int nz, float rx, float ry, float rz, float sx, float sy, float sz,
                                int taper, float* __restrict__ out) {
  const long total = (long)nx * ny * nz;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((long)nx * ny));
    const float vx = __fdiv_rn(__fsub_rn((float)(x - nx / 2), sx), rx);
    const float vy = __fdiv_rn(__fsub_rn((float)(y - ny / 2), sy), ry);
    const float vz = __fdiv_rn(__fsub_rn((float)(z - nz / 2), sz), rz);
    const float q = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
    float v = q <= 1.f ? 1.f : 0.f;
    if (x < taper || y < taper || x >= nx - taper || y >= ny - taper || (nz > 1 && (z < taper || z >= nz - taper)))
      v = 0.f;
    out[i] = v;
  }
}

// MASK ./ max(MASK); MASK(MASK <= 0.001) = 0
__global__ void k_mask_normalise(float* __restrict__ v, long n, const unsigned* __restrict__ keys) {
  const float mx = key_to_float(keys[1]);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float r = v[i] / mx;
    v[i] = r <= 0.001f ? 0.f : r;
  }
}

// Separable convolution of v (in place through `tmp`) with the same 1-D taps along x, y and z.
emc_status conv3(float* v, float* tmp, int nx, int ny, int nz, const Taps& t, int blocks, cudaStream_t st) {
  k_conv_axis<<<blocks, 256, 0, st>>>(v, tmp, nx, ny, nz, 0, t);
  k_conv_axis<<<blocks, 256, 0, st>>>(tmp, v, nx, ny, nz, 1, t);
  k_conv_axis<<<blocks, 256, 0, st>>>(v, tmp, nx, ny, nz, 2, t);
  EMC_LAUNCH_CHECK();
  EMC_CUDA(cudaMemcpyAsync(v, tmp, sizeof(float) * (size_t)nx * ny * nz, cudaMemcpyDeviceToDevice, st));
  return EMC_OK;
}

int grid_blocks(long total) { return (int)std::max<long>(1, std::min<long>((total + 255) / 256, 8L * device_sm_count())); }

// ------------------------------------------------------------------ cubic splines (host, FP64)
// The interpolating cubic spline with not-a-knot end conditions (the spline through the data that
// MATLAB's fit(x, y, 'cubicSpline') and spline() build), as piecewise polynomials
// p_j(x) = y_j + b_j t + c_j t^2 + d_j t^3, t = x - x_j.  Slopes s_j solve the tridiagonal system of
// continuous second derivatives, with the first and last rows enforcing a continuous third
// derivative at x_1 and x_{n-2}.
struct Spline {
  std::vector<double> x, a, b, c, d;
};

// Tridiagonal solve by Gaussian elimination with partial pivoting (row swaps bring in a second
// super-diagonal).  dl: sub-diagonal (n-1), dg: diagonal (n), du: super-diagonal (n-1); rhs is
// overwritten by the solution.  Returns false on a zero pivot.
bool solve_tridiagonal(std::vector<double> dl, std::vector<double> dg, std::vector<double> du, std::vector<double>& rhs) {
  const int n = (int)dg.size();
  std::vector<double> du2(std::max(n - 2, 0), 0.0);
  for (int i = 0; i + 1 < n; ++i) {
    if (std::fabs(dg[i]) >= std::fabs(dl[i])) {
      if (dg[i] == 0.0) return false;
      const double f = dl[i] / dg[i];
      dg[i + 1] -= f * du[i];
      rhs[i + 1] -= f * rhs[i];
    } else {
      // swap rows i and i+1
      const double f = dg[i] / dl[i];
      dg[i] = dl[i];
      const double t = dg[i + 1];
      dg[i + 1] = du[i] - f * t;
      if (i + 2 < n) {
        du2[i] = du[i + 1];
        du[i + 1] = -f * du2[i];
      }
      du[i] = t;
      const double r = rhs[i];
      rhs[i] = rhs[i + 1];
      rhs[i + 1] = r - f * rhs[i + 1];
    }
  }
  if (dg[n - 1] == 0.0) return false;
  rhs[n - 1] /= dg[n - 1];
  if (n > 1) rhs[n - 2] = (rhs[n - 2] - du[n - 2] * rhs[n - 1]) / dg[n - 2];
  for (int i = n - 3; i >= 0; --i) rhs[i] = (rhs[i] - du[i] * rhs[i + 1] - du2[i] * rhs[i + 2]) / dg[i];
  return true;
}

bool make_spline(const std::vector<double>& x, const std::vector<double>& y, Spline& s) {
  const int n = (int)x.size();
  s.x = x;
  s.a = y;
  s.b.assign(std::max(n - 1, 1), 0.0);
  s.c.assign(std::max(n - 1, 1), 0.0);
  s.d.assign(std::max(n - 1, 1), 0.0);
  if (n == 1) return true;
  std::vector<double> dx(n - 1), m(n - 1);
  for (int i = 0; i + 1 < n; ++i) {
    dx[i] = x[i + 1] - x[i];
    if (!(dx[i] > 0.0)) return false;
    m[i] = (y[i + 1] - y[i]) / dx[i];
  }
  if (n == 2) {
    s.b[0] = m[0];
    return true;
  }
  if (n == 3) {
    // not-a-knot with three points: the parabola through them
    const double c2 = (m[1] - m[0]) / (x[2] - x[0]);
    s.b[0] = m[0] - c2 * dx[0];
    s.c[0] = c2;
    s.b[1] = s.b[0] + 2.0 * c2 * dx[0];
    s.c[1] = c2;
    return true;
  }
  std::vector<double> dl(n - 1), dg(n), du(n - 1), r(n);
  dg[0] = dx[1];
  du[0] = dx[0] + dx[1];
  r[0] = ((dx[0] + 2.0 * du[0]) * dx[1] * m[0] + dx[0] * dx[0] * m[1]) / du[0];
  for (int i = 1; i + 1 < n; ++i) {
    dl[i - 1] = dx[i];
    dg[i] = 2.0 * (dx[i - 1] + dx[i]);
    du[i] = dx[i - 1];
    r[i] = 3.0 * (dx[i] * m[i - 1] + dx[i - 1] * m[i]);
  }
  const double e = dx[n - 2] + dx[n - 3];
  dl[n - 2] = e;
  dg[n - 1] = dx[n - 3];
  r[n - 1] = (dx[n - 2] * dx[n - 2] * m[n - 3] + (2.0 * e + dx[n - 2]) * dx[n - 3] * m[n - 2]) / e;
  if (!solve_tridiagonal(dl, dg, du, r)) return false;
  for (int j = 0; j + 1 < n; ++j) {
    s.b[j] = r[j];
    s.c[j] = (3.0 * m[j] - 2.0 * r[j] - r[j + 1]) / dx[j];
    s.d[j] = (r[j] + r[j + 1] - 2.0 * m[j]) / (dx[j] * dx[j]);
  }
  return true;
}

// Piecewise evaluation; outside [x_0, x_{n-1}] the end pieces extrapolate (as ppval does).
__host__ __device__ inline double spline_eval(const double* x, const double* a, const double* b, const double* c,
                                              const double* d, int n, double v) {
  if (n == 1) return a[0];
  int lo = 0, hi = n - 2;
  while (lo < hi) {  // largest j in [0, n-2] with x_j <= v
    const int mid = (lo + hi + 1) / 2;
    if (x[mid] <= v) lo = mid; else hi = mid - 1;
  }
  const double t = v - x[lo];
  return a[lo] + t * (b[lo] + t * (c[lo] + t * d[lo]));
}

// cRef(|k|) on the half spectrum in FFT order; the radius is formed in single precision as the
// reference's single radialGrid (BH_multi_gridCoordinates(.., 1, 0, 1) ./ pixelSize) and the
// spline is evaluated in FP64.
__global__ void k_cref_eval(int nx, int ny, int nz, float pixel, const double* __restrict__ coef, int n,
                            float* __restrict__ out) {
  const int nh = nx / 2 + 1;
  const long total = (long)nh * ny * nz;
  const double *x = coef, *a = coef + n, *b = coef + 2 * n, *c = coef + 3 * n, *d = coef + 4 * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int kx = (int)(i % nh);
    const int q = (int)((i / nh) % ny), r = (int)(i / ((long)nh * ny));
    const int ky = q <= ny / 2 ? q : q - ny, kz = r <= nz / 2 ? r : r - nz;
    const float fx = (float)kx / (float)nx, fy = (float)ky / (float)ny, fz = (float)kz / (float)nz;
    const float rad = sqrtf(fx * fx + fy * fy + fz * fz) / pixel;
    out[i] = (float)spline_eval(x, a, b, c, d, n, (double)rad);
  }
}

// ifftshift of `count` centred volumes, keeping the half spectrum: out[v][r][q][p] (p <= nx/2) =
// in[v][(r + cz) % nz][(q + cy) % ny][(p + cx) % nx] with c = floor(n/2) per axis.
__global__ void k_centred_to_half(const float* __restrict__ in, int nx, int ny, int nz, long count,
                                  float* __restrict__ out) {
  const int nh = nx / 2 + 1;
  const long per = (long)nh * ny * nz, nv = (long)nx * ny * nz;
  const long total = per * count;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long v = i / per, j = i % per;
    const int p = (int)(j % nh), q = (int)((j / nh) % ny), r = (int)(j / ((long)nh * ny));
    out[i] = in[v * nv + ((long)((r + nz / 2) % nz) * ny + (q + ny / 2) % ny) * nx + (p + nx / 2) % nx];
  }
}

}  // namespace
}  // namespace emc

extern "C" {

emc_status emc_centred_to_half(const float* d_in, int nx, int ny, int nz, int count, float* d_out, void* stream) {
  using namespace emc;
  EMC_CHECK_ARG(d_in && d_out && nx > 0 && ny > 0 && nz > 0 && count >= 0, "emc_centred_to_half: bad argument");
  EMC_CHECK_ARG(d_in != d_out, "emc_centred_to_half: in place is not supported");
  if (count == 0) return EMC_OK;
  const long total = (long)(nx / 2 + 1) * ny * nz * count;
  k_centred_to_half<<<grid_blocks(total), 256, 0, as_stream(stream)>>>(d_in, nx, ny, nz, count, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_binary_wedge(int n, float tilt_min_deg, float tilt_max_deg, int smooth, int layout, float* d_out,
                            void* stream) {
  using namespace emc;
  EMC_CHECK_ARG(d_out && n >= 8 && n <= 1024, "emc_binary_wedge: bad argument (n = %d)", n);
  EMC_CHECK_ARG(tilt_min_deg <= tilt_max_deg, "emc_binary_wedge: tilt_min > tilt_max");
  EMC_CHECK_ARG(layout == 0 || layout == 1, "emc_binary_wedge: layout %d", layout);
  cudaStream_t st = as_stream(stream);
  const long total = (long)n * n * n;
  const int blocks = grid_blocks(total);
  // maxTilt = 90 - |min(tilts)|, minTilt = 90 - |max(tilts)| (BH_weightMask3d.m:109-110)
  const double max_cone = 90.0 - std::fabs((double)tilt_min_deg), min_cone = 90.0 - std::fabs((double)tilt_max_deg);
  float* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, sizeof(float) * (2 * total + 2), st));
  float* a = buf;
  float* b = buf + total;
  unsigned* keys = reinterpret_cast<unsigned*>(buf + 2 * total);
  emc_status rs = EMC_OK;
  k_wedge_binary<<<blocks, 256, 0, st>>>(n, max_cone, min_cone, a);
  if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  if (rs == EMC_OK && smooth) {
    // BH_multi_gaussian3d(9, 1.5): the normalised separable Gaussian on -4..4
    Taps t{};
    t.len = 9;
    double sum = 0.0;
    double w[9];
    for (int k = 0; k < 9; ++k) sum += (w[k] = std::exp(-0.5 * ((k - 4) / 1.5) * ((k - 4) / 1.5)));
    for (int k = 0; k < 9; ++k) t.w[k] = (float)(w[k] / sum);
    rs = conv3(a, b, n, n, n, t, blocks, st);
  }
  if (rs == EMC_OK) {
    k_times_nyquist<<<blocks, 256, 0, st>>>(a, n);
    if (cudaMemsetAsync(keys, 0xff, sizeof(unsigned), st) != cudaSuccess ||
        cudaMemsetAsync(keys + 1, 0, sizeof(unsigned), st) != cudaSuccess)
      rs = EMC_E_CUDA;
    k_minmax<<<blocks, 256, 0, st>>>(a, total, keys);
    k_wedge_normalise<<<blocks, 256, 0, st>>>(a, n, keys, layout, d_out);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  cudaFreeAsync(buf, st);
  if (rs != EMC_OK) set_error("emc_binary_wedge: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return rs;
}

emc_status emc_mask_sphere(const int size[3], const double radius[3], const double shift[3], double kernel_frac,
                           float* d_out, void* stream) {
  using namespace emc;
  EMC_CHECK_ARG(size && radius && d_out, "emc_mask_sphere: null argument");
  EMC_CHECK_ARG(size[0] > 1 && size[1] > 1 && size[2] >= 1, "emc_mask_sphere: size");
  EMC_CHECK_ARG(radius[0] > 1 && radius[1] > 1 && (size[2] == 1 || radius[2] > 1),
                "emc_mask_sphere: every radius must be > 1 (EMC_maskShape checkIN)");
  EMC_CHECK_ARG(kernel_frac >= 0.0 && kernel_frac <= 1.0, "emc_mask_sphere: kernel fraction %g", kernel_frac);
  cudaStream_t st = as_stream(stream);
  const int nx = size[0], ny = size[1], nz = size[2];
  const long total = (long)nx * ny * nz;
  const int blocks = grid_blocks(total);
  const bool blur = kernel_frac > 0.0;
  int k = 0;
  Taps t{};
  if (blur) {
    // kernelSize = round((min(SIZE) * kernel - 1) / 2) * 2 + 1, at least 9; sigma keeps the Gaussian
    // at 0.5 half way through the roll-off (EMC_maskShape.m:99-107)
    const int mn = nz > 1 ? std::min(nx, std::min(ny, nz)) : std::min(nx, ny);
    k = (int)std::round((mn * kernel_frac - 1.0) / 2.0) * 2 + 1;
    if (k < 9) k = 9;
    EMC_CHECK_ARG(k <= kMaxTaps, "emc_mask_sphere: kernel of %d taps (at most %d)", k, kMaxTaps);
    const int m = (k + 1) / 2;
    EMC_CHECK_ARG(nx >= 2 * m + 1 && ny >= 2 * m + 1 && (nz == 1 || nz >= 2 * m + 1),
                  "emc_mask_sphere: with a kernel of %d the minimum size is %d", k, 2 * m + 1);
    const double middle = m / 2.0;
    const double sigma = std::sqrt(-middle * middle / (2.0 * std::log(0.5)));
    // EMC_gaussianKernel([1, k], sigma): exp(-0.5 (v / sigma)^2) on v = -(k-1)/2 .. (k-1)/2, sum 1,
    // in single precision
    float w[kMaxTaps];
    float sum = 0.f;
    for (int j = 0; j < k; ++j) {
      const float v = (float)(j - (k - 1) / 2) / (float)sigma;
      w[j] = std::exp(-0.5f * v * v);
      sum += w[j];
    }
    t.len = k;
    for (int j = 0; j < k; ++j) t.w[j] = w[j] / sum;
  }
  const int taper = blur ? (k + 1) / 2 : 0;
  const float rx = (float)(radius[0] + taper), ry = (float)(radius[1] + taper),
              rz = (float)((nz > 1 ? radius[2] : 1.0) + (nz > 1 ? taper : 0));
  const float sx = shift ? (float)shift[0] : 0.f, sy = shift ? (float)shift[1] : 0.f,
              sz = shift && nz > 1 ? (float)shift[2] : 0.f;
  k_sphere_binary<<<blocks, 256, 0, st>>>(nx, ny, nz, rx, ry, nz > 1 ? rz : 1e30f, sx, sy, sz, taper, d_out);
  EMC_LAUNCH_CHECK();
  if (!blur) return EMC_OK;
  float* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, sizeof(float) * (total + 2), st));
  unsigned* keys = reinterpret_cast<unsigned*>(buf + total);
  emc_status rs = EMC_OK;
  if (nz > 1) {
    rs = conv3(d_out, buf, nx, ny, nz, t, blocks, st);
  } else {
    k_conv_axis<<<blocks, 256, 0, st>>>(d_out, buf, nx, ny, 1, 0, t);
    k_conv_axis<<<blocks, 256, 0, st>>>(buf, d_out, nx, ny, 1, 1, t);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK) {
    if (cudaMemsetAsync(keys, 0xff, sizeof(unsigned), st) != cudaSuccess ||
        cudaMemsetAsync(keys + 1, 0, sizeof(unsigned), st) != cudaSuccess)
      rs = EMC_E_CUDA;
    k_minmax<<<blocks, 256, 0, st>>>(d_out, total, keys);
    k_mask_normalise<<<blocks, 256, 0, st>>>(d_out, total, keys);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  cudaFreeAsync(buf, st);
  if (rs != EMC_OK) set_error("emc_mask_sphere: launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return rs;
}

emc_status emc_cref_filter(const double* shell_freq, const double* shell_fsc, int n_shells, const double* os_freq,
                           const double* force_mask, int n_os, double mtf, const int size[3], float pixel_size,
                           float* d_out, void* stream) {
  using namespace emc;
  EMC_CHECK_ARG(shell_freq && shell_fsc && os_freq && size && d_out && n_shells >= 2 && n_os >= 2 && n_os <= 1 << 20,
                "emc_cref_filter: bad argument");
  EMC_CHECK_ARG(size[0] >= 1 && size[1] >= 1 && size[2] >= 1 && pixel_size > 0.f, "emc_cref_filter: size / pixel");
  // fitFSC = fit(shells, max(FSC, 0), 'cubicSpline') (BH_multi_cRef.m:62-65)
  std::vector<double> xs(shell_freq, shell_freq + n_shells), ys(n_shells);
  for (int i = 0; i < n_shells; ++i) ys[i] = shell_fsc[i] > 0.0 ? shell_fsc[i] : 0.0;
  Spline fsc;
  EMC_CHECK_ARG(make_spline(xs, ys, fsc), "emc_cref_filter: shell frequencies must increase strictly");
  // the ad hoc MTF of fscINFO{3}{3} (:102-139) on the oversampled axis
  std::vector<double> ox(os_freq, os_freq + n_os), oy(n_os);
  for (int i = 0; i < n_os; ++i) {
    double m = 1.0;
    if (mtf != 0.0) {
      double det, cap;
      if (mtf == 1.0) {
        det = -100.0;
        cap = 0.05;
      } else if (mtf == 2.0) {
        det = -25.0;
        cap = 0.06;
      } else {
        det = -std::round(mtf);
        cap = mtf - std::round(mtf);
      }
      m = 1.0 / ((std::exp(det * std::pow(ox[i], 1.25)) + cap) / cap);
    }
    const double f = spline_eval(fsc.x.data(), fsc.a.data(), fsc.b.data(), fsc.c.data(), fsc.d.data(), n_shells, ox[i]);
    // cRef = fit(osX, sqrt(abs(2 F ./ (1 + F))) .* adHocMTF .* forceMask, 'cubicSpline') (:142-143)
    oy[i] = std::sqrt(std::fabs(2.0 * f / (1.0 + f))) * m * (force_mask ? force_mask[i] : 1.0);
  }
  Spline cref;
  EMC_CHECK_ARG(make_spline(ox, oy, cref), "emc_cref_filter: oversampled frequencies must increase strictly");
  std::vector<double> packed(5 * (size_t)n_os, 0.0);
  for (int i = 0; i < n_os; ++i) {
    packed[i] = cref.x[i];
    packed[n_os + i] = cref.a[i];
    if (i + 1 < n_os) {
      packed[2 * n_os + i] = cref.b[i];
      packed[3 * n_os + i] = cref.c[i];
      packed[4 * n_os + i] = cref.d[i];
    }
  }
  cudaStream_t st = as_stream(stream);
  double* coef = nullptr;
  EMC_CUDA(cudaMallocAsync(&coef, sizeof(double) * packed.size(), st));
  emc_status rs = EMC_OK;
  if (cudaMemcpyAsync(coef, packed.data(), sizeof(double) * packed.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
    rs = EMC_E_CUDA;
  const long total = (long)(size[0] / 2 + 1) * size[1] * size[2];
  if (rs == EMC_OK) {
    k_cref_eval<<<grid_blocks(total), 256, 0, st>>>(size[0], size[1], size[2], pixel_size, coef, n_os, d_out);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  cudaFreeAsync(coef, st);
  // the coefficient table is pageable host memory: wait for its copy before it goes out of scope
  if (rs == EMC_OK && cudaStreamSynchronize(st) != cudaSuccess) rs = EMC_E_CUDA;
  if (rs != EMC_OK) set_error("emc_cref_filter: %s", cudaGetErrorString(cudaGetLastError()));
  return rs;
}

}  // extern "C"
