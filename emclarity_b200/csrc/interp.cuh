// interp.cuh -- trilinear / tricubic samplers shared by the rotation kernels.
//
// Index-space convention (reference mexFiles/mexXform3d.cu:45-74, :293-296): output voxel p
// samples the source at s = M (p - c - t) + c ('forward') or s = M (p - c) + t + c ('inv'),
// c = floor(n/2).  The reference reaches the same point through normalised texture
// coordinates (t + size_shift)/n + 0.5; in index space that is exactly s above.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace emc {

// FP32 -> BF16 (round to nearest even) copy of a device array (defined in xform3d.cu).
emc_status to_bf16(const float* in, __nv_bfloat16* out, long n, cudaStream_t st);

template <typename T>
__device__ __forceinline__ float ldv(const T* p, long i);
template <>
__device__ __forceinline__ float ldv<float>(const float* p, long i) { return __ldg(p + i); }
template <>
__device__ __forceinline__ float ldv<__nv_bfloat16>(const __nv_bfloat16* p, long i) {
  return __bfloat162float(p[i]);
}

// Trilinear with interpn(...,'linear',0) semantics: 0 unless 0 <= s <= n-1 on every axis.
template <typename T>
__device__ __forceinline__ float sample_linear(const T* __restrict__ v, int nx, int ny, int nz, float sx, float sy,
                                               float sz) {
  if (!(sx >= 0.f && sy >= 0.f && sz >= 0.f && sx <= (float)(nx - 1) && sy <= (float)(ny - 1) &&
        sz <= (float)(nz - 1)))
    return 0.f;
  const int x0 = min((int)sx, nx - 1), y0 = min((int)sy, ny - 1), z0 = min((int)sz, nz - 1);
  const float fx = sx - (float)x0, fy = sy - (float)y0, fz = sz - (float)z0;
  const int x1 = min(x0 + 1, nx - 1), y1 = min(y0 + 1, ny - 1), z1 = min(z0 + 1, nz - 1);
  const long pz0 = (long)z0 * ny, pz1 = (long)z1 * ny;
  const float c000 = ldv(v, (pz0 + y0) * nx + x0), c100 = ldv(v, (pz0 + y0) * nx + x1);
  const float c010 = ldv(v, (pz0 + y1) * nx + x0), c110 = ldv(v, (pz0 + y1) * nx + x1);
  const float c001 = ldv(v, (pz1 + y0) * nx + x0), c101 = ldv(v, (pz1 + y0) * nx + x1);
  const float c011 = ldv(v, (pz1 + y1) * nx + x0), c111 = ldv(v, (pz1 + y1) * nx + x1);
  const float c00 = fmaf(fx, c100 - c000, c000), c10 = fmaf(fx, c110 - c010, c010);
  const float c01 = fmaf(fx, c101 - c001, c001), c11 = fmaf(fx, c111 - c011, c011);
  const float c0 = fmaf(fy, c10 - c00, c00), c1 = fmaf(fy, c11 - c01, c01);
  return fmaf(fz, c1 - c0, c0);
}

template <typename T>
__device__ __forceinline__ float vox_or_zero(const T* v, int nx, int ny, int nz, int x, int y, int z) {
  return (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) ? ldv(v, ((long)z * ny + y) * nx + x) : 0.f;
}

// Trilinear with zero-valued voxels around the volume: the cudaAddressModeBorder behaviour
// of the reference texture (mexXform3d.cu:269-271), evaluated with FP32 weights.
template <typename T>
__device__ __forceinline__ float sample_linear_border(const T* __restrict__ v, int nx, int ny, int nz, float sx,
                                                      float sy, float sz) {
  if (!(sx > -1.f && sy > -1.f && sz > -1.f && sx < (float)nx && sy < (float)ny && sz < (float)nz)) return 0.f;
  const float fx0 = floorf(sx), fy0 = floorf(sy), fz0 = floorf(sz);
  const int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
  const float fx = sx - fx0, fy = sy - fy0, fz = sz - fz0;
  float acc = 0.f;
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
        acc = fmaf(w, vox_or_zero(v, nx, ny, nz, x0 + dx, y0 + dy, z0 + dz), acc);
      }
  return acc;
}

// Catmull-Rom (Keys a = -1/2) cubic convolution weights for taps at offsets -1, 0, 1, 2.
__host__ __device__ __forceinline__ void catmull_rom(float t, float w[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (-t3 + 2.f * t2 - t);
  w[1] = 0.5f * (3.f * t3 - 5.f * t2 + 2.f);
  w[2] = 0.5f * (-3.f * t3 + 4.f * t2 + t);
  w[3] = 0.5f * (t3 - t2);
}
__host__ __device__ __forceinline__ void catmull_rom_d(float t, float w[4]) {
  const float t2 = t * t;
  w[0] = 0.5f * (-3.f * t2 + 4.f * t - 1.f);
  w[1] = 0.5f * (9.f * t2 - 10.f * t);
  w[2] = 0.5f * (-9.f * t2 + 8.f * t + 1.f);
  w[3] = 0.5f * (3.f * t2 - 2.f * t);
}

// Tricubic, zero outside [0, n-1] and zero-valued voxels beyond the edges.
template <typename T>
__device__ __forceinline__ float sample_cubic(const T* __restrict__ v, int nx, int ny, int nz, float sx, float sy,
                                              float sz) {
  if (!(sx >= 0.f && sy >= 0.f && sz >= 0.f && sx <= (float)(nx - 1) && sy <= (float)(ny - 1) &&
        sz <= (float)(nz - 1)))
    return 0.f;
  const int x0 = (int)sx, y0 = (int)sy, z0 = (int)sz;
  float wx[4], wy[4], wz[4];
  catmull_rom(sx - (float)x0, wx);
  catmull_rom(sy - (float)y0, wy);
  catmull_rom(sz - (float)z0, wz);
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float accy = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float accx = 0.f;
#pragma unroll
      for (int i = 0; i < 4; ++i) accx = fmaf(wx[i], vox_or_zero(v, nx, ny, nz, x0 - 1 + i, y0 - 1 + j, z0 - 1 + k), accx);
      accy = fmaf(wy[j], accx, accy);
    }
    acc = fmaf(wz[k], accy, acc);
  }
  return acc;
}

// Value and gradient (d/dsx, d/dsy, d/dsz) of the tricubic interpolant.
template <typename T>
__device__ __forceinline__ float sample_cubic_grad(const T* __restrict__ v, int nx, int ny, int nz, float sx, float sy,
                                                   float sz, float g[3]) {
  g[0] = g[1] = g[2] = 0.f;
  if (!(sx >= 0.f && sy >= 0.f && sz >= 0.f && sx <= (float)(nx - 1) && sy <= (float)(ny - 1) &&
        sz <= (float)(nz - 1)))
    return 0.f;
  const int x0 = (int)sx, y0 = (int)sy, z0 = (int)sz;
  float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
  catmull_rom(sx - (float)x0, wx); catmull_rom_d(sx - (float)x0, dx);
  catmull_rom(sy - (float)y0, wy); catmull_rom_d(sy - (float)y0, dy);
  catmull_rom(sz - (float)z0, wz); catmull_rom_d(sz - (float)z0, dz);
  float val = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    float a = 0.f, ax = 0.f, ay = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      float b = 0.f, bx = 0.f;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float c = vox_or_zero(v, nx, ny, nz, x0 - 1 + i, y0 - 1 + j, z0 - 1 + k);
        b = fmaf(wx[i], c, b);
        bx = fmaf(dx[i], c, bx);
      }
      a = fmaf(wy[j], b, a);
      ax = fmaf(wy[j], bx, ax);
      ay = fmaf(dy[j], b, ay);
    }
    val = fmaf(wz[k], a, val);
    gx = fmaf(wz[k], ax, gx);
    gy = fmaf(wz[k], ay, gy);
    gz = fmaf(dz[k], a, gz);
  }
  g[0] = gx; g[1] = gy; g[2] = gz;
  return val;
}

template <typename T>
__device__ __forceinline__ float sample(int mode, const T* __restrict__ v, int nx, int ny, int nz, float sx, float sy,
                                        float sz) {
  return mode == EMC_INTERP_CUBIC ? sample_cubic(v, nx, ny, nz, sx, sy, sz)
       : mode == EMC_INTERP_LINEAR_BORDER ? sample_linear_border(v, nx, ny, nz, sx, sy, sz)
                                          : sample_linear(v, nx, ny, nz, sx, sy, sz);
}

}  // namespace emc
