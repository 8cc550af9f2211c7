// ctf.cu -- 2-D CTF images (mexCTF replacement) and the 3-D CTF^2 sampling-function wedge
// (mexSF3D replacement).
//
// Reference: mexFiles/include/core_headers.cuh:40-81 (ctfParams), mexFiles/utils/ctf.cu:12-130
// (kernels), mexFiles/mexCTF.cu:6-121, mexFiles/mexSF3D.cu:24-302.  The reference builds the
// SF3D volume with one texture upload and one launch per tilt; here all tilt images are made
// by one launch and a second launch accumulates every tilt into each (x, y) column.
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace emc {

struct CtfDev {
  float cs_term, df_term, amp_phase, df1, df2, ast;
};

// ctfParams(doHalfGrid, doSqCTF, pix, lambda, Cs, AC, df1, df2, ast) evaluated in float on the
// host like the reference's __host__ constructor (core_headers.cuh:63-75).
static CtfDev make_ctf(const emc_ctf_params& p) {
  const float PI = 3.14159265358979323f;
  CtfDev c;
  c.amp_phase = atanf(p.amp_contrast / sqrtf(1.0f - p.amp_contrast * p.amp_contrast));
  c.df1 = 0.5f * (p.defocus1 + p.defocus2);
  c.df2 = 0.5f * (p.defocus1 - p.defocus2);
  c.ast = p.astig_deg * PI / 180.0f - (PI * (float)lrintf(p.astig_deg / 180.0f));
  c.cs_term = PI * 0.5f * p.cs_mm * 1e7f * (p.wavelength * p.wavelength * p.wavelength);
  c.df_term = PI * p.wavelength;
  return c;
}

struct CtfGrid {
  int dx, ny;      // output width (nx/2+1 or nx) and height
  int ox, oy;      // origin used by the centred / wrapped coordinate mapping
  int half, centred, squared;
  float fvx, fvy;  // Fourier voxel size 1/(pix*nx), 1/(pix*ny)
};

__device__ __forceinline__ float ctf_eval(const CtfDev& c, const CtfGrid& g, int x0, int y0, int* xs) {
  int x = x0, y = y0;
  if (g.centred) {
    y -= g.oy;
    if (!g.half) x -= g.ox;
  } else {
    if (y > g.oy) y -= g.ny;
    if (!g.half && x > g.ox) x -= g.dx;
  }
  *xs = x;
  const float fy = (float)y * g.fvy;
  const float fx = (float)x * g.fvx;
  const float phi = atan2f(fy, fx);
  const float r2 = fx * fx + fy * fy;
  const float v = sinf(c.cs_term * (r2 * r2) - c.df_term * r2 * (c.df1 + c.df2 * cosf(2.0f * (phi - c.ast))) -
                       c.amp_phase);
  return g.squared ? v * v : v;
}

// plain (ctf.cu:12-66) and exposure-filtered (ctf.cu:68-130) CTF images
__global__ void k_ctf2d(const CtfDev c, const CtfGrid g, int use_exposure, float radial_weight, float exposure,
                        float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= g.dx || y >= g.ny) return;
  int xs;
  float v = ctf_eval(c, g, x, y, &xs);
  if (use_exposure) {
    const float rw = radial_weight * (xs == 0 ? 0.2f : fabsf((float)xs));
    int ys = y;
    if (g.centred) ys -= g.oy; else if (ys > g.oy) ys -= g.ny;
    const float fx = (float)xs * g.fvx, fy = (float)ys * g.fvy;
    const float r2 = fx * fx + fy * fy;
    // Grant-Grigorieff critical exposure a*s^(2b)+c with a = 0.24499, b = -0.8325 (on s^2), c = 2.8141
    v *= rw * expf((-0.5f * exposure) / (0.24499f * powf(r2, -0.8325f) + 2.81410f));
  }
  out[(long)y * g.dx + x] = v;
}

// All tilt images of the SF3D weight (full grid, centred, squared, exposure-filtered) of a batch of
// volumes: image blockIdx.z = p * ntilts + t uses the CTF c[blockIdx.z] (volume p, tilt t) and tilt
// t's grid, occupancy and exposure.
__global__ void k_sf3d_ctfs(const CtfDev* __restrict__ c, const CtfGrid* __restrict__ g, const float* __restrict__ occ,
                            const float* __restrict__ expo, int nx, int ny, int ntilts, float* __restrict__ imgs) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int t = blockIdx.z % ntilts;
  if (x >= nx || y >= ny) return;
  int xs;
  const CtfGrid gg = g[t];
  float v = ctf_eval(c[blockIdx.z], gg, x, y, &xs);
  const float rw = occ[t] * (xs == 0 ? 0.2f : fabsf((float)xs));
  const int ys = y - gg.oy;
  const float fx = (float)xs * gg.fvx, fy = (float)ys * gg.fvy;
  const float r2 = fx * fx + fy * fy;
  v *= rw * expf((-0.5f * expo[t]) / (0.24499f * powf(r2, -0.8325f) + 2.81410f));
  imgs[((long)blockIdx.z * ny + y) * nx + x] = v;
}

// sf3dKernel (mexSF3D.cu:24-78) summed over tilts: for every (x, y) column and tilt, the voxels
// within 4 px of the tilted central plane receive the bilinearly sampled CTF^2 image (zero
// border) times the cosine edge weight.  Volume blockIdx.z of a batch: its images follow those of
// the previous volumes, its output volume too.
__global__ void k_sf3d_accum(const float* __restrict__ imgs, const float2* __restrict__ sincos, int ntilts, int nx,
                             int ny, int nz, float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= nx || y >= ny) return;
  imgs += (long)blockIdx.z * ntilts * nx * ny;
  out += (long)blockIdx.z * nx * ny * nz;
  const float PI = 3.14159265358979323f;
  const float ssx = (nx % 2 == 0) ? 0.5f : 0.f, ssy = (ny % 2 == 0) ? 0.5f : 0.f, ssz = (nz % 2 == 0) ? 0.5f : 0.f;
  const float u = (float)x - (float)nx / 2.0f;
  const float tv = ((float)(y - ny / 2) + ssy) / (float)ny + 0.5f;
  const float ty = tv * (float)ny - 0.5f;
  for (int t = 0; t < ntilts; ++t) {
    const float sA = sincos[t].x, cA = sincos[t].y;
    const float tw_pre = -u * sA + ssz;
    const float* img = imgs + (long)t * nx * ny;
    for (int z = 0; z < nz; ++z) {
      const float w = (float)(z - nz / 2);
      const float tw = tw_pre + w * cA;
      if (tw < -4.0f || tw > 4.0f) continue;
      const float zw = (0.5f + 0.5f * cosf(tw * (PI / 4.0f))) * 0.25f;
      float tu = u * cA + w * sA + ssx;
      tu = tu / (float)nx + 0.5f;
      const float tx = tu * (float)nx - 0.5f;
      const float fx0 = floorf(tx), fy0 = floorf(ty);
      const int x0 = (int)fx0, y0 = (int)fy0;
      const float fx = tx - fx0, fy = ty - fy0;
      float acc = 0.f;
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx) {
          const int xi = x0 + dx, yi = y0 + dy;
          if (xi < 0 || yi < 0 || xi >= nx || yi >= ny) continue;
          acc += (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * img[(long)yi * nx + xi];
        }
      out[((long)z * ny + y) * nx + x] += zw * acc;
    }
  }
}

// Binary Y-tilt-axis missing wedge of masking/BH_weightMask3d.m:103-120 on the half spectrum
// (FFT order, the ifftshift of the reference's centred grid), without the Gaussian smoothing
// (emc_binary_wedge applies it): theta = atan2d(kx, kz) is excluded inside the
// +/-(90 - tilt) cones around kz; the |kx|,|kz| <= 2 slab through the origin is kept; times the
// 'nyquist' radial window of BH_bandpass3d (:124-131 of BH_weightMask3d.m).  Optionally times the 3-D CTF of |k|
// (ctf.cu:45-62 with the radius taken in 3-D).
__global__ void k_wedge_ctf(int n, float max_cone, float min_cone, int use_ctf, int squared, const CtfDev c,
                            float inv_box_pix, float* __restrict__ out) {
  const int nh = n / 2 + 1;
  const long total = (long)nh * n * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    // signed frequencies of the ifftshifted centred grid: for even n the Nyquist index is -n/2
    const int kx0 = (int)(i % nh);
    const int ky0 = (int)((i / nh) % n), kz0 = (int)(i / ((long)nh * n));
    const int kx = 2 * kx0 < n ? kx0 : kx0 - n;
    const int ky = 2 * ky0 < n ? ky0 : ky0 - n;
    const int kz = 2 * kz0 < n ? kz0 : kz0 - n;
    const float theta = atan2f((float)kx, (float)kz) * (180.0f / 3.14159265358979323f);
    const bool excluded = (180.0f - min_cone <= theta || theta <= max_cone - 180.0f) ||
                          (-min_cone <= theta && theta <= max_cone);
    float w = excluded ? 0.f : 1.f;
    if (abs(kx) <= 2 && abs(kz) <= 2) w = 1.f;
    const float r2i = (float)(kx * kx + ky * ky + kz * kz);
    // BH_bandpass3d(size, 0, 0, 0, METHOD, 'nyquist'): 1 below 0.485 cycles/pixel, Gaussian
    // roll-off of width 1.5/n beyond (masking/BH_bandpass3d.m:60-77, :88-92)
    const float rn = sqrtf(r2i) / (float)n;
    if (rn >= 0.485f) {
      const float roll = 1.5f / (float)n;
      w *= expf(-(rn - 0.485f) * (rn - 0.485f) / (2.f * roll * roll));
    }
    if (use_ctf && w != 0.f) {
      const float r2 = r2i * inv_box_pix * inv_box_pix;
      const float v = sinf(c.cs_term * (r2 * r2) - c.df_term * r2 * c.df1 - c.amp_phase);
      w *= squared ? v * v : v;
    }
    out[i] = w;
  }
}

static CtfGrid make_grid(int nx, int ny, int half, int squared, int centred, float pix) {
  CtfGrid g;
  g.half = half;
  g.centred = centred;
  g.squared = squared;
  g.ny = ny;
  g.dx = half ? nx / 2 + 1 : nx;
  g.ox = half ? 0 : nx / 2;
  g.oy = ny / 2;
  g.fvx = 1.0f / (pix * (float)nx);
  g.fvy = 1.0f / (pix * (float)ny);
  return g;
}

// Per-volume minimum (for SF3D - (min(SF3D(:)) - 1e-4), masking/BH_weightMaskMex.m:55).
__global__ void k_vol_min(const float* __restrict__ v, long n, unsigned* __restrict__ out_key) {
  __shared__ unsigned red[32];
  const float* src = v + (long)blockIdx.y * n;
  unsigned best = 0xffffffffu;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float x = src[i];
    // order-preserving key of a float; NaN sorts last
    const unsigned u = __float_as_uint(x);
    const unsigned k = (x != x) ? 0xffffffffu : ((u & 0x80000000u) ? ~u : (u | 0x80000000u));
    best = min(best, k);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned b = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = min(b, red[w]);
    atomicMin(out_key + blockIdx.y, b);
  }
}

__global__ void k_vol_sub_min(float* __restrict__ v, long n, const unsigned* __restrict__ key, float eps) {
  float* dst = v + (long)blockIdx.y * n;
  const unsigned k = key[blockIdx.y];
  const unsigned u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  const float mn = __uint_as_float(u);
  const float off = mn - eps;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = dst[i] - off;
}

}  // namespace emc

extern "C" {

emc_status emc_ctf2d(const emc_ctf_params* p, int nx, int ny, int half, int squared, int centred, float* d_out,
                     void* stream) {
  EMC_CHECK_ARG(p && d_out, "emc_ctf2d: null argument");
  EMC_CHECK_ARG(nx > 0 && ny > 0, "emc_ctf2d: bad size");
  EMC_CHECK_ARG(p->pixel_size > 0.f && p->amp_contrast >= 0.f && p->amp_contrast < 1.f, "emc_ctf2d: bad parameters");
  const emc::CtfDev c = emc::make_ctf(*p);
  const emc::CtfGrid g = emc::make_grid(nx, ny, half, squared, centred, p->pixel_size);
  dim3 block(32, 8), grid((g.dx + 31) / 32, (ny + 7) / 8);
  emc::k_ctf2d<<<grid, block, 0, emc::as_stream(stream)>>>(c, g, 0, 0.f, 0.f, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_ctf2d_exposure(const emc_ctf_params* p, int nx, int ny, int half, int squared, int centred,
                              float radial_weight, float total_exposure, float* d_out, void* stream) {
  EMC_CHECK_ARG(p && d_out, "emc_ctf2d_exposure: null argument");
  EMC_CHECK_ARG(nx > 0 && ny > 0, "emc_ctf2d_exposure: bad size");
  const emc::CtfDev c = emc::make_ctf(*p);
  const emc::CtfGrid g = emc::make_grid(nx, ny, half, squared, centred, p->pixel_size);
  dim3 block(32, 8), grid((g.dx + 31) / 32, (ny + 7) / 8);
  emc::k_ctf2d<<<grid, block, 0, emc::as_stream(stream)>>>(c, g, 1, radial_weight, total_exposure, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_wedge_ctf_weight(int n, float tilt_min_deg, float tilt_max_deg, const emc_ctf_params* ctf,
                                int squared, float* d_out, void* stream) {
  EMC_CHECK_ARG(d_out && n >= 2, "emc_wedge_ctf_weight: bad argument");
  EMC_CHECK_ARG(tilt_min_deg <= tilt_max_deg, "emc_wedge_ctf_weight: tilt_min > tilt_max");
  // maxTilt = 90 - |min(tilts)|, minTilt = 90 - |max(tilts)| (BH_weightMask3d.m:109-110)
  const float max_cone = 90.0f - fabsf(tilt_min_deg), min_cone = 90.0f - fabsf(tilt_max_deg);
  emc::CtfDev c{};
  float inv_box_pix = 0.f;
  if (ctf) {
    EMC_CHECK_ARG(ctf->pixel_size > 0.f, "emc_wedge_ctf_weight: pixel size");
    c = emc::make_ctf(*ctf);
    inv_box_pix = 1.0f / ((float)n * ctf->pixel_size);
  }
  const long total = (long)(n / 2 + 1) * n * n;
  const int blocks = (int)std::min<long>((total + 255) / 256, 4L * emc::device_sm_count());
  emc::k_wedge_ctf<<<blocks, 256, 0, emc::as_stream(stream)>>>(n, max_cone, min_cone, ctf ? 1 : 0, squared, c,
                                                                inv_box_pix, d_out);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_sf3d(int half, int squared, const unsigned size[3], const float* pix, const float* wavelength,
                    const float* cs_mm, const float* df1, const float* df2, const float* astig_deg,
                    const float* amp_contrast, unsigned n_tilts, const float* tilt_deg, const float* exposure,
                    const float* occupancy, float* d_out, void* stream) {
  EMC_CHECK_ARG(size && pix && wavelength && cs_mm && df1 && df2 && astig_deg && amp_contrast && tilt_deg &&
                    exposure && occupancy && d_out,
                "emc_sf3d: null argument");
  EMC_CHECK_ARG(half == 0, "emc_sf3d: only the full grid is built (as in the reference)");
  EMC_CHECK_ARG(n_tilts > 0 && n_tilts < 100000, "emc_sf3d: n_tilts %u", n_tilts);
  const int nx = (int)size[0], ny = (int)size[1], nz = (int)size[2];
  EMC_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "emc_sf3d: bad size");
  cudaStream_t st = emc::as_stream(stream);
  std::vector<emc::CtfDev> cs(n_tilts);
  std::vector<emc::CtfGrid> gs(n_tilts);
  std::vector<float2> sc(n_tilts);
  for (unsigned t = 0; t < n_tilts; ++t) {
    emc_ctf_params p{pix[t], wavelength[t], cs_mm[t], amp_contrast[t], df1[t], df2[t], astig_deg[t]};
    cs[t] = emc::make_ctf(p);
    gs[t] = emc::make_grid(nx, ny, 0, squared, 1, pix[t]);
    // sincosf(deg_2_rad(-tilt)) (mexSF3D.cu:131-135)
    const float a = -tilt_deg[t] * 3.14159265358979323f / 180.0f;
    sc[t] = make_float2(sinf(a), cosf(a));
  }
  const size_t img_bytes = sizeof(float) * (size_t)n_tilts * nx * ny;
  const size_t hdr_bytes = (sizeof(emc::CtfDev) + sizeof(emc::CtfGrid) + sizeof(float2) + 2 * sizeof(float)) * n_tilts;
  char* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, img_bytes + hdr_bytes + 256, st));
  float* imgs = reinterpret_cast<float*>(buf);
  char* q = buf + ((img_bytes + 15) / 16) * 16;
  emc::CtfDev* d_c = reinterpret_cast<emc::CtfDev*>(q);
  q += sizeof(emc::CtfDev) * n_tilts;
  emc::CtfGrid* d_g = reinterpret_cast<emc::CtfGrid*>(q);
  q += sizeof(emc::CtfGrid) * n_tilts;
  q = reinterpret_cast<char*>(((uintptr_t)q + 7) & ~(uintptr_t)7);
  float2* d_sc = reinterpret_cast<float2*>(q);
  q += sizeof(float2) * n_tilts;
  float* d_occ = reinterpret_cast<float*>(q);
  float* d_exp = d_occ + n_tilts;
  emc_status rs = EMC_OK;
  if (cudaMemcpyAsync(d_c, cs.data(), sizeof(emc::CtfDev) * n_tilts, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_g, gs.data(), sizeof(emc::CtfGrid) * n_tilts, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_sc, sc.data(), sizeof(float2) * n_tilts, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_occ, occupancy, sizeof(float) * n_tilts, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_exp, exposure, sizeof(float) * n_tilts, cudaMemcpyHostToDevice, st) ||
      cudaMemsetAsync(d_out, 0, sizeof(float) * (size_t)nx * ny * nz, st)) {
    emc::set_error("emc_sf3d: upload failed");
    rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK) {
    dim3 block(32, 8), grid((nx + 31) / 32, (ny + 7) / 8, n_tilts);
    emc::k_sf3d_ctfs<<<grid, block, 0, st>>>(d_c, d_g, d_occ, d_exp, nx, ny, (int)n_tilts, imgs);
    dim3 grid2((nx + 31) / 32, (ny + 7) / 8);
    emc::k_sf3d_accum<<<grid2, block, 0, st>>>(imgs, d_sc, (int)n_tilts, nx, ny, nz, d_out);
    if (cudaGetLastError() != cudaSuccess) {
      emc::set_error("emc_sf3d: launch failed");
      rs = EMC_E_CUDA;
    }
  }
  // host staging vectors must outlive the async copies
  cudaStreamSynchronize(st);
  cudaFreeAsync(buf, st);
  return rs;
}

// BH_weightMaskMex(SIZE, SAMPLING, TLT, xyzSubTomo, reconGeometry) for a batch of particles
// (masking/BH_weightMaskMex.m:1-60), arithmetic in single precision like the reference (TLT is cast to
// single first, :11).
emc_status emc_sf3d_particles(const unsigned size[3], double sampling, const double* tlt, int rows, int cols,
                              const double* xyz, const double recon_geometry[6], int count, float* d_out,
                              void* stream) {
  EMC_CHECK_ARG(size && tlt && xyz && recon_geometry && d_out, "emc_sf3d_particles: null argument");
  EMC_CHECK_ARG(rows > 0 && cols >= 19, "emc_sf3d_particles: tilt table %d x %d (needs 19 columns)", rows, cols);
  EMC_CHECK_ARG(count >= 0, "emc_sf3d_particles: count %d", count);
  if (count == 0) return EMC_OK;
  // sortrows(TLT, 1): stable ascending sort on column 1, then single precision
  std::vector<int> order(rows);
  for (int r = 0; r < rows; ++r) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return tlt[(size_t)a * cols] < tlt[(size_t)b * cols]; });
  auto T = [&](int r, int c) { return (float)tlt[(size_t)order[r] * cols + (c - 1)]; };  // 1-based column
  const int n = rows;
  std::vector<float> pix(n), lam(n), cs(n), ac(n), def0(n), ddf(n), dphi(n), tilt(n), expo(n), occ(n);
  float dose_mean = 0.f;
  for (int r = 0; r < n; ++r) dose_mean += T(r, 14);
  dose_mean /= (float)n;
  std::vector<float> elastic(n);
  float el_max = 0.f;
  for (int r = 0; r < n; ++r) {
    pix[r] = T(r, 16) * (float)sampling * 1e10f;
    cs[r] = T(r, 17) * 1e3f;
    lam[r] = T(r, 18) * 1e10f;
    ac[r] = T(r, 19);
    def0[r] = -T(r, 15) * 1e10f;
    ddf[r] = T(r, 12) * 1e10f;
    dphi[r] = T(r, 13) * 180.0f / 3.14159265358979323846f;
    tilt[r] = T(r, 4);
    expo[r] = T(r, 11);
    // fractionOfElastics = exp(-thickness / (cosd(tilt) * 400)), thickness 75 nm, normalised (:44-46)
    elastic[r] = expf(-75.0f / (cosf(tilt[r] * 3.14159265358979323846f / 180.0f) * 400.0f));
    el_max = std::max(el_max, elastic[r]);
  }
  for (int r = 0; r < n; ++r) occ[r] = (elastic[r] / el_max) * (T(r, 14) / dose_mean);
  // originVol = ceil((reconGeometry(1, 1:3) + 1) / 2), reconShift = reconGeometry(2, :) (:17-20)
  double origin[3], rshift[3];
  for (int d = 0; d < 3; ++d) {
    origin[d] = ceil((recon_geometry[d] + 1.0) / 2.0);
    rshift[d] = recon_geometry[3 + d];
  }
  const long nv = (long)size[0] * size[1] * size[2];
  const int nx = (int)size[0], ny = (int)size[1], nz = (int)size[2];
  EMC_CHECK_ARG(nx > 0 && ny > 0 && nz > 0 && n < 65536, "emc_sf3d_particles: bad size or tilt count");
  cudaStream_t st = emc::as_stream(stream);
  // every (particle, tilt) CTF, with the particle's defocus offset by its height along the beam
  std::vector<emc::CtfDev> cs_all((size_t)count * n);
  for (int p = 0; p < count; ++p) {
    const double v[3] = {xyz[3 * (size_t)p] - origin[0] + rshift[0], xyz[3 * (size_t)p + 1] - origin[1] + rshift[1],
                         xyz[3 * (size_t)p + 2] - origin[2] + rshift[2]};
    for (int r = 0; r < n; ++r) {
      // rTilt = defineMatrix(tilt, 'TILT', 'forwardVector') = [c 0 s; 0 1 0; -s 0 c]; z of rTilt * v (:27-30)
      const float a = tilt[r] * (3.14159265358979323846f / 180.0f);
      const float z = -sinf(a) * (float)v[0] + cosf(a) * (float)v[2];
      const float d = def0[r] - z * pix[r];
      const emc_ctf_params cp{pix[r], lam[r], cs[r], ac[r], d + ddf[r], d - ddf[r], dphi[r]};
      cs_all[(size_t)p * n + r] = emc::make_ctf(cp);
    }
  }
  std::vector<emc::CtfGrid> gs(n);
  std::vector<float2> sc(n);
  for (int r = 0; r < n; ++r) {
    gs[r] = emc::make_grid(nx, ny, 0, 1, 1, pix[r]);
    const float a = -tilt[r] * 3.14159265358979323f / 180.0f;  // sincosf(deg_2_rad(-tilt)) (mexSF3D.cu:131-135)
    sc[r] = make_float2(sinf(a), cosf(a));
  }
  // particles per launch pair: the tilt images of a chunk stay under 1 GiB, and the image grid's z
  // extent (particles x tilts) under 65536
  const size_t img_per = sizeof(float) * (size_t)n * nx * ny;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>({(size_t)count, (size_t)(65535 / n),
                                                               (size_t)(1ull << 30) / img_per}));
  const size_t c_bytes = sizeof(emc::CtfDev) * cs_all.size();
  const size_t hdr = ((c_bytes + sizeof(emc::CtfGrid) * n + 15) / 16) * 16 + sizeof(float2) * n + 2 * sizeof(float) * n;
  char* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, img_per * chunk + hdr + 256, st));
  float* imgs = reinterpret_cast<float*>(buf);
  char* q = buf + ((img_per * chunk + 15) / 16) * 16;
  emc::CtfDev* d_c = reinterpret_cast<emc::CtfDev*>(q);
  emc::CtfGrid* d_g = reinterpret_cast<emc::CtfGrid*>(q + c_bytes);
  q += ((c_bytes + sizeof(emc::CtfGrid) * n + 15) / 16) * 16;
  float2* d_sc = reinterpret_cast<float2*>(q);
  float* d_occ = reinterpret_cast<float*>(d_sc + n);
  float* d_exp = d_occ + n;
  emc_status rs0 = EMC_OK;
  if (cudaMemcpyAsync(d_c, cs_all.data(), c_bytes, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_g, gs.data(), sizeof(emc::CtfGrid) * n, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_sc, sc.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_occ, occ.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st) ||
      cudaMemcpyAsync(d_exp, expo.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st) ||
      cudaMemsetAsync(d_out, 0, sizeof(float) * (size_t)nv * count, st)) {
    emc::set_error("emc_sf3d_particles: upload failed");
    rs0 = EMC_E_CUDA;
  }
  dim3 block(32, 8);
  for (int p0 = 0; p0 < count && rs0 == EMC_OK; p0 += chunk) {
    const int cnt = std::min(chunk, count - p0);
    emc::k_sf3d_ctfs<<<dim3((nx + 31) / 32, (ny + 7) / 8, cnt * n), block, 0, st>>>(d_c + (size_t)p0 * n, d_g, d_occ,
                                                                                     d_exp, nx, ny, n, imgs);
    emc::k_sf3d_accum<<<dim3((nx + 31) / 32, (ny + 7) / 8, cnt), block, 0, st>>>(imgs, d_sc, n, nx, ny, nz,
                                                                                 d_out + (size_t)p0 * nv);
    if (cudaGetLastError() != cudaSuccess) {
      emc::set_error("emc_sf3d_particles: launch failed");
      rs0 = EMC_E_CUDA;
    }
  }
  // the host tables must outlive their copies
  if (cudaStreamSynchronize(st) != cudaSuccess && rs0 == EMC_OK) rs0 = EMC_E_CUDA;
  cudaFreeAsync(buf, st);
  EMC_TRY(rs0);
  // SF3D - (min(SF3D(:)) - 1e-4) (:55)
  unsigned* keys = nullptr;
  EMC_CUDA(cudaMallocAsync((void**)&keys, sizeof(unsigned) * count, st));
  emc_status rs = EMC_OK;
  if (cudaMemsetAsync(keys, 0xff, sizeof(unsigned) * count, st) != cudaSuccess) rs = EMC_E_CUDA;
  const int gx = (int)std::max<long>(1, std::min<long>((nv + 255) / 256, 64));
  for (int p0 = 0; p0 < count && rs == EMC_OK; p0 += 65535) {
    const int cnt = std::min(65535, count - p0);
    emc::k_vol_min<<<dim3(gx, cnt), 256, 0, st>>>(d_out + (size_t)p0 * nv, nv, keys + p0);
    emc::k_vol_sub_min<<<dim3(gx, cnt), 256, 0, st>>>(d_out + (size_t)p0 * nv, nv, keys + p0, 1e-4f);
    if (cudaGetLastError() != cudaSuccess) rs = EMC_E_CUDA;
  }
  if (rs == EMC_E_CUDA) emc::set_error("emc_sf3d_particles: %s", cudaGetErrorString(cudaGetLastError()));
  cudaFreeAsync(keys, st);
  return rs;
}

}  // extern "C"
