// average.cu -- subtomogram averaging: the accumulation loop of BH_average3d.
//
// Reference: transformations/BH_average3d.m:1207-1500.  For every (particle, peak) the loop
//   * rotates the extracted window back with interpolator(..., angles, shift, 'inv', symmetry)
//     (:1417; testScripts/interpolator.m:29-78 -- the sum over symmetry copies A * S_k, divided
//     by their number; mexFiles/mexXform3d.cu:45-74 texture trilinear with a zero border),
//   * rotates its wedge / CTF weight the same way with a zero shift (:1429),
//   * normalises inside the binary mask  interpMask > 0.01  (:1087-1092, :1439-1441):
//       r = (r - mean(r(B))) / rms(r(B) - mean) .* interpMask,
//   * drops the particle when mean(r(:)) is not finite (:1450-1456),
//   * adds r .* peakWgt and w .* peakWgt to the sums of its half set (:1462-1482),
// and the half-set average is sum / count (:1703-1707).
//
// B200 layout: a batch of particles is rotated into a scratch slab [batch][n^3] (8^3 output
// bricks per CTA, 4x4x2 voxel tiles per warp, FP64 statistics per particle reduced with one atomic
// per block), a per-particle kernel turns the statistics into (mean, rms, keep), and an
// output-stationary pass adds the batch to the half-set sums voxel by voxel in the reference's
// particle order (so the FP32 sums round the same way whatever the batch split).  No atomics touch
// the sums: results are deterministic.
#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "interp.cuh"

namespace emc {

constexpr int kAvgMaxSym = 60;

struct AvgParticle {
  float shift[3];
  float weight;  // peakWgt
  int half;      // 1 odd, 2 even
  int wedge;     // index into the wedge volumes, -1 none
  int nsym;
  int pad;
};

struct AvgStats {
  double s1, s2;  // sum and sum of squares over the binary mask
  double s3;      // sum of r * mask over all voxels (finite check)
};

struct AvgCoef {
  float mean, rms;
  int keep;
  int pad;
};

// Zero-border trilinear sample (cudaAddressModeBorder of the reference texture) with the same
// weights and summation order as sample_linear_border -- bit-identical results -- but with the
// eight loads unchecked when the whole cell lies inside the volume (almost every sample).
__device__ __forceinline__ float avg_sample_border(const float* __restrict__ v, int n, float sx, float sy, float sz) {
  if (!(sx > -1.f && sy > -1.f && sz > -1.f && sx < (float)n && sy < (float)n && sz < (float)n)) return 0.f;
  const float fx0 = floorf(sx), fy0 = floorf(sy), fz0 = floorf(sz);
  const int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
  const float fx = sx - fx0, fy = sy - fy0, fz = sz - fz0;
  if (x0 < 0 || y0 < 0 || z0 < 0 || x0 >= n - 1 || y0 >= n - 1 || z0 >= n - 1)
    return sample_linear_border(v, n, n, n, sx, sy, sz);
  const float* b = v + ((long)z0 * n + y0) * n + x0;
  const long sy_ = n, sz_ = (long)n * n;
  const float c[8] = {__ldg(b), __ldg(b + 1), __ldg(b + sy_), __ldg(b + sy_ + 1),
                      __ldg(b + sz_), __ldg(b + sz_ + 1), __ldg(b + sz_ + sy_), __ldg(b + sz_ + sy_ + 1)};
  float acc = 0.f;
#pragma unroll
  for (int dz = 0; dz < 2; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
        acc = fmaf(w, c[4 * dz + 2 * dy + dx], acc);
      }
  return acc;
}

// Sampling point of output voxel (x, y, z) under matrix m (rows), 'inv' direction:
// s = M (p - c) + t + c (mexXform3d.cu:58-66), the same arithmetic as k_xform3d.
__device__ __forceinline__ float avg_sample(const float* __restrict__ src, int n, const float* m, float u, float v,
                                            float w, const float* t, int c) {
  float sx = fmaf(m[0], u, fmaf(m[1], v, m[2] * w));
  float sy = fmaf(m[3], u, fmaf(m[4], v, m[5] * w));
  float sz = fmaf(m[6], u, fmaf(m[7], v, m[8] * w));
  sx += t[0];
  sy += t[1];
  sz += t[2];
  return avg_sample_border(src, n, sx + (float)c, sy + (float)c, sz + (float)c);
}

// Rotates particle blockIdx.y of the batch into out[blockIdx.y]; with `mask`, accumulates the
// particle's statistics.  mats: [batch][kAvgMaxSym][9] rows of A * S_k.  One CTA per 8^3 output
// brick (blockIdx.x), each warp on a 4x4x2 voxel tile, two voxels per thread: a rotated 4x4x2
// tile reads a compact source neighbourhood, so the warp's 256 corner loads touch far fewer
// sectors than a rotated 32-voxel row would.  Symmetry copies are summed in operator order.
constexpr int kBrick = 8;

__global__ void __launch_bounds__(256) k_avg_rotate(const float* __restrict__ vols, long vol_stride,
                                                          const int* __restrict__ vol_index, int n,
                                                          const float* __restrict__ mats,
                                                          const AvgParticle* __restrict__ parts, int use_shift,
                                                          const float* __restrict__ mask, float bin_thr,
                                                          float* __restrict__ out, AvgStats* __restrict__ stats) {
  __shared__ double red[3][32];
  const int p = blockIdx.y;
  const AvgParticle pr = parts[p];
  const int vi = vol_index ? vol_index[p] : p;
  const long nv = (long)n * n * n;
  float* dst = out + (long)p * nv;
  const int nb = (n + kBrick - 1) / kBrick;
  const int b = blockIdx.x;
  const int t = threadIdx.x;
  const int x = (b % nb) * kBrick + ((t & 3) | (((t >> 5) & 1) << 2));
  const int y = ((b / nb) % nb) * kBrick + (((t >> 2) & 3) | (((t >> 6) & 1) << 2));
  const int zb = (b / (nb * nb)) * kBrick + (((t >> 4) & 1) | (((t >> 7) & 1) << 1));
  const int c = n / 2;
  const float zero[3] = {0.f, 0.f, 0.f};
  const float* sh = use_shift ? pr.shift : zero;
  const float* src = vols + (long)(vi < 0 ? 0 : vi) * vol_stride;
  const float* m0 = mats + (long)p * kAvgMaxSym * 9;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int z = zb + 4 * q;
    if (x >= n || y >= n || z >= n) continue;
    const long i = ((long)z * n + y) * n + x;
    float r = 0.f;
    if (vi >= 0) {
      const float u = (float)(x - c), v = (float)(y - c), w = (float)(z - c);
      float acc = 0.f;
      for (int k = 0; k < pr.nsym; ++k) acc += avg_sample(src, n, m0 + 9 * k, u, v, w, sh, c);
      r = pr.nsym > 1 ? acc / (float)pr.nsym : acc;
    }
    dst[i] = r;
    if (mask && vi >= 0) {
      const float mk = __ldg(mask + i);
      if (mk > bin_thr) {
        s1 += (double)r;
        s2 += (double)r * (double)r;
      }
      s3 += (double)r * (double)mk;
    }
  }
  if (!mask) return;
  const int lane = t & 31, warp = t >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    s3 += __shfl_xor_sync(0xffffffffu, s3, off);
  }
  if (lane == 0) {
    red[0][warp] = s1;
    red[1][warp] = s2;
    red[2][warp] = s3;
  }
  __syncthreads();
  if (t == 0) {
    double t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) {
      t1 += red[0][wi];
      t2 += red[1][wi];
      t3 += red[2][wi];
    }
    atomicAdd(&stats[p].s1, t1);
    atomicAdd(&stats[p].s2, t2);
    atomicAdd(&stats[p].s3, t3);
  }
}

// Copies a batch's parameters from the mapped host staging into device memory (the symmetry
// matrices of each particle, its AvgParticle record and its wedge index).
__global__ void k_avg_stage_in(const float* __restrict__ mats_h, const AvgParticle* __restrict__ parts_h,
                               const int* __restrict__ widx_h, int nb, int nsym, float* __restrict__ mats,
                               AvgParticle* __restrict__ parts, int* __restrict__ widx) {
  const int per = 9 * nsym;
  const long total = (long)nb * per;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const long i = t / per, r = t % per;
    mats[i * kAvgMaxSym * 9 + r] = mats_h[i * kAvgMaxSym * 9 + r];
  }
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nb; i += (long)gridDim.x * blockDim.x) {
    parts[i] = parts_h[i];
    widx[i] = widx_h[i];
  }
}

// mean / rms inside the binary mask and the finite check of mean(r_normalised(:)); counts the
// kept particles of each half set.
__global__ void k_avg_coef(const AvgStats* __restrict__ stats, const AvgParticle* __restrict__ parts, int count,
                           double n_bin, double mask_sum, double n_vox, AvgCoef* __restrict__ coef,
                           unsigned long long* __restrict__ half_count, int* __restrict__ kept) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= count) return;
  const AvgStats s = stats[p];
  const double mean = s.s1 / n_bin;
  const double var = s.s2 / n_bin - mean * mean;
  const double rms = sqrt(var > 0.0 ? var : 0.0);
  // mean over all voxels of (r - mean) / rms .* mask
  const double trim = (s.s3 - mean * mask_sum) / (rms * n_vox);
  const int keep = isfinite(trim) && rms > 0.0 && (parts[p].half == 1 || parts[p].half == 2) ? 1 : 0;
  AvgCoef c;
  c.mean = (float)mean;
  c.rms = (float)rms;
  c.keep = keep;
  c.pad = 0;
  coef[p] = c;
  kept[p] = keep;
  if (keep) atomicAdd(&half_count[parts[p].half - 1], 1ull);
}

// Adds the batch to the half-set sums, voxel by voxel, particles in order.
// particle term: ((r - mean) / rms) * mask * weight;  wedge term: w * weight.
__global__ void __launch_bounds__(256) k_avg_accumulate(const float* __restrict__ rot, long nv, int count,
                                                        const AvgCoef* __restrict__ coef,
                                                        const AvgParticle* __restrict__ parts,
                                                        const float* __restrict__ mask, int normalise,
                                                        float* __restrict__ sum_odd, float* __restrict__ sum_even) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* s_c = reinterpret_cast<float4*>(smem_raw);  // (mean, rms, weight, half | 0 when dropped)
  for (int p = threadIdx.x; p < count; p += blockDim.x) {
    const AvgCoef c = coef[p];
    const AvgParticle pr = parts[p];
    s_c[p] = make_float4(c.mean, c.rms, pr.weight, c.keep ? (float)pr.half : 0.f);
  }
  __syncthreads();
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nv; i += (long)gridDim.x * blockDim.x) {
    float a1 = sum_odd[i], a2 = sum_even[i];
    const float mk = normalise ? __ldg(mask + i) : 1.f;
    // groups of U particles: all U loads in flight, then added in order
    constexpr int U = 8;
    for (int p0 = 0; p0 < count; p0 += U) {
      float r[U];
#pragma unroll
      for (int u = 0; u < U; ++u) r[u] = (p0 + u < count) ? __ldg(rot + (long)(p0 + u) * nv + i) : 0.f;
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (p0 + u >= count) break;
        const float4 c = s_c[p0 + u];
        if (c.w == 0.f) continue;
        float t;
        if (normalise) {
          t = __fdiv_rn(r[u] - c.x, c.y);
          t = t * mk;
        } else {
          t = r[u];
        }
        t = t * c.z;
        if (c.w == 1.f)
          a1 += t;
        else
          a2 += t;
      }
    }
    sum_odd[i] = a1;
    sum_even[i] = a2;
  }
}

// avgVolume = avgVolume ./ nExtracted (BH_average3d.m:1705-1706), correctly rounded.
__global__ void k_avg_finish(const float* __restrict__ sum, long nv, float count, float* __restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nv; i += (long)gridDim.x * blockDim.x)
    out[i] = __fdiv_rn(sum[i], count);
}

__global__ void k_avg_mask_stats(const float* __restrict__ mask, long nv, float thr, double* __restrict__ out) {
  __shared__ double red[2][32];
  double nb = 0.0, ms = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nv; i += (long)gridDim.x * blockDim.x) {
    const float m = mask[i];
    nb += m > thr ? 1.0 : 0.0;
    ms += (double)m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nb += __shfl_xor_sync(0xffffffffu, nb, o);
    ms += __shfl_xor_sync(0xffffffffu, ms, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = nb;
    red[1][warp] = ms;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    atomicAdd(&out[0], a);
    atomicAdd(&out[1], b);
  }
}

}  // namespace emc

struct emc_average_s {
  int n = 0, nw = 0;
  long nv = 0, nvw = 0;
  float* mask = nullptr;
  float bin_thr = 0.01f;
  double n_bin = 0.0, mask_sum = 0.0;
  int nsym = 1;
  std::vector<double> sym;  // [nsym][9] column-major
  float* sum[2] = {nullptr, nullptr};
  float* wsum[2] = {nullptr, nullptr};
  unsigned long long* counts = nullptr;  // [2]
  int batch = 0;
  float* rot = nullptr;    // [batch][nv]
  float* wrot = nullptr;   // [batch][nvw]
  float* mats = nullptr;   // [batch][kAvgMaxSym][9]
  emc::AvgParticle* parts = nullptr;
  emc::AvgStats* stats = nullptr;
  emc::AvgCoef* coef = nullptr;
  int* kept = nullptr;
  int* widx = nullptr;
  // Per-batch parameters (mats, parts, widx, in that order) staged in pinned host memory mapped into
  // the device's address space: a kernel pulls them into mats / parts / widx over PCIe, so they take
  // no copy-engine slot behind a caller's large host-to-device copy on another stream.
  unsigned char* h_stage = nullptr;
  const unsigned char* d_stage = nullptr;
};

namespace {

void avg_free(emc_average_s* a) {
  cudaFree(a->mask);
  for (int h = 0; h < 2; ++h) {
    cudaFree(a->sum[h]);
    cudaFree(a->wsum[h]);
  }
  cudaFree(a->counts);
  cudaFree(a->rot);
  cudaFree(a->wrot);
  cudaFree(a->mats);
  cudaFree(a->parts);
  cudaFree(a->stats);
  cudaFree(a->coef);
  cudaFree(a->kept);
  cudaFree(a->widx);
  if (a->h_stage) cudaFreeHost(a->h_stage);
}

size_t stage_bytes(int batch) {
  return (sizeof(float) * 9 * emc::kAvgMaxSym + sizeof(emc::AvgParticle) + sizeof(int)) * (size_t)batch;
}

int grid_for(long n) { return (int)std::max<long>(1, std::min<long>((n + 255) / 256, 8L * emc::device_sm_count())); }

}  // namespace

extern "C" {

emc_status emc_average_create(int n, const float* d_mask, float bin_threshold, int nw, const double* sym, int nsym,
                              int batch, emc_average_t* out, void* stream) {
  EMC_CHECK_ARG(out && d_mask, "emc_average_create: null argument");
  *out = nullptr;
  EMC_CHECK_ARG(n >= 2 && n <= 1024, "emc_average_create: box %d", n);
  EMC_CHECK_ARG(nw >= 0 && nw <= 1024, "emc_average_create: wedge box %d", nw);
  EMC_CHECK_ARG(nsym >= 1 && nsym <= emc::kAvgMaxSym, "emc_average_create: nsym %d not in 1..%d", nsym,
                emc::kAvgMaxSym);
  EMC_CHECK_ARG(nsym == 1 || sym, "emc_average_create: %d symmetry matrices but none given", nsym);
  emc_average_s* a = new (std::nothrow) emc_average_s();
  EMC_CHECK_ARG(a, "emc_average_create: host allocation failed");
  a->n = n;
  a->nw = nw;
  a->nv = (long)n * n * n;
  a->nvw = (long)nw * nw * nw;
  a->bin_thr = bin_threshold;
  a->nsym = nsym;
  a->sym.assign(9 * (size_t)nsym, 0.0);
  if (sym) {
    std::copy(sym, sym + 9 * nsym, a->sym.begin());
  } else {
    a->sym[0] = a->sym[4] = a->sym[8] = 1.0;
  }
  const size_t per = sizeof(float) * ((size_t)a->nv + (size_t)a->nvw);
  a->batch = batch > 0 ? batch : (int)std::max<size_t>(1, std::min<size_t>(4096, (1ull << 31) / per));
  cudaStream_t st = emc::as_stream(stream);
  emc_status rs = EMC_OK;
  auto alloc = [&](void** p, size_t bytes) {
    if (rs == EMC_OK && cudaMalloc(p, std::max<size_t>(bytes, 4)) != cudaSuccess) {
      emc::set_error("emc_average_create: cudaMalloc(%zu) failed", bytes);
      rs = EMC_E_OOM;
    }
  };
  alloc((void**)&a->mask, sizeof(float) * a->nv);
  for (int h = 0; h < 2; ++h) {
    alloc((void**)&a->sum[h], sizeof(float) * a->nv);
    if (nw) alloc((void**)&a->wsum[h], sizeof(float) * a->nvw);
  }
  alloc((void**)&a->counts, 2 * sizeof(unsigned long long));
  alloc((void**)&a->rot, sizeof(float) * a->nv * a->batch);
  if (nw) alloc((void**)&a->wrot, sizeof(float) * a->nvw * a->batch);
  alloc((void**)&a->mats, sizeof(float) * 9 * emc::kAvgMaxSym * a->batch);
  alloc((void**)&a->parts, sizeof(emc::AvgParticle) * a->batch);
  alloc((void**)&a->stats, sizeof(emc::AvgStats) * a->batch);
  alloc((void**)&a->coef, sizeof(emc::AvgCoef) * a->batch);
  alloc((void**)&a->kept, sizeof(int) * a->batch);
  alloc((void**)&a->widx, sizeof(int) * a->batch);
  if (rs == EMC_OK) {
    void* dp = nullptr;
    if (cudaHostAlloc((void**)&a->h_stage, stage_bytes(a->batch), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&dp, a->h_stage, 0) != cudaSuccess) {
      emc::set_error("emc_average_create: mapped host staging (%zu bytes) failed", stage_bytes(a->batch));
      rs = EMC_E_OOM;
    }
    a->d_stage = reinterpret_cast<const unsigned char*>(dp);
  }
  double* d_ms = nullptr;
  alloc((void**)&d_ms, 2 * sizeof(double));
  if (rs == EMC_OK) {
    double h_ms[2] = {0.0, 0.0};
    if (cudaMemcpyAsync(a->mask, d_mask, sizeof(float) * a->nv, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(d_ms, 0, 2 * sizeof(double), st) != cudaSuccess) {
      rs = EMC_E_CUDA;
    } else {
      emc::k_avg_mask_stats<<<grid_for(a->nv), 256, 0, st>>>(a->mask, a->nv, a->bin_thr, d_ms);
      if (cudaGetLastError() != cudaSuccess ||
          cudaMemcpyAsync(h_ms, d_ms, sizeof(h_ms), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess)
        rs = EMC_E_CUDA;
    }
    if (rs == EMC_E_CUDA) emc::set_error("emc_average_create: %s", cudaGetErrorString(cudaGetLastError()));
    a->n_bin = h_ms[0];
    a->mask_sum = h_ms[1];
    if (rs == EMC_OK && a->n_bin < 1.0) {
      emc::set_error("emc_average_create: no mask voxel above %g", (double)bin_threshold);
      rs = EMC_E_ARG;
    }
  }
  cudaFree(d_ms);
  if (rs == EMC_OK) rs = emc_average_reset(a, stream);
  if (rs != EMC_OK) {
    avg_free(a);
    delete a;
    return rs;
  }
  *out = a;
  return EMC_OK;
}

emc_status emc_average_reset(emc_average_t a, void* stream) {
  EMC_CHECK_ARG(a, "emc_average_reset: null handle");
  cudaStream_t st = emc::as_stream(stream);
  for (int h = 0; h < 2; ++h) {
    EMC_CUDA(cudaMemsetAsync(a->sum[h], 0, sizeof(float) * a->nv, st));
    if (a->nw) EMC_CUDA(cudaMemsetAsync(a->wsum[h], 0, sizeof(float) * a->nvw, st));
  }
  EMC_CUDA(cudaMemsetAsync(a->counts, 0, 2 * sizeof(unsigned long long), st));
  return EMC_OK;
}

emc_status emc_average_add(emc_average_t a, const float* d_particles, int count, const double* rot,
                           const float* shift, const float* weight, const int* half, const float* d_wedges,
                           int n_wedges, const int* wedge_index, int* kept, void* stream) {
  EMC_CHECK_ARG(a && rot && half, "emc_average_add: null argument");
  EMC_CHECK_ARG(count >= 0, "emc_average_add: count %d", count);
  if (count == 0) return EMC_OK;
  EMC_CHECK_ARG(d_particles, "emc_average_add: null particles");
  EMC_CHECK_ARG(!a->nw || (d_wedges && wedge_index && n_wedges > 0),
                "emc_average_add: the handle averages wedges; give the wedge volumes and indices");
  for (int p = 0; p < count; ++p) {
    EMC_CHECK_ARG(half[p] == 1 || half[p] == 2, "emc_average_add: particle %d half set %d (must be 1 or 2)", p,
                  half[p]);
    if (a->nw)
      EMC_CHECK_ARG(wedge_index[p] >= 0 && wedge_index[p] < n_wedges, "emc_average_add: particle %d wedge %d", p,
                    wedge_index[p]);
  }
  cudaStream_t st = emc::as_stream(stream);
  // host views of the mapped staging (every batch ends with a stream synchronisation, so the
  // device has read a batch's parameters before the next batch overwrites them)
  float* mats = reinterpret_cast<float*>(a->h_stage);
  emc::AvgParticle* parts = reinterpret_cast<emc::AvgParticle*>(a->h_stage + sizeof(float) * 9 * emc::kAvgMaxSym *
                                                                                (size_t)a->batch);
  int* widx = reinterpret_cast<int*>(parts + a->batch);
  const float* d_mats_h = reinterpret_cast<const float*>(a->d_stage);
  const emc::AvgParticle* d_parts_h = reinterpret_cast<const emc::AvgParticle*>(
      a->d_stage + sizeof(float) * 9 * emc::kAvgMaxSym * (size_t)a->batch);
  const int* d_widx_h = reinterpret_cast<const int*>(d_parts_h + a->batch);
  std::vector<int> kept_h(a->batch);
  for (int b0 = 0; b0 < count; b0 += a->batch) {
    const int nb = std::min(a->batch, count - b0);
    for (int i = 0; i < nb; ++i) {
      const int p = b0 + i;
      const double* A = rot + 9 * (size_t)p;  // column-major 3x3
      for (int k = 0; k < a->nsym; ++k) {
        const double* S = a->sym.data() + 9 * k;
        float* m = mats + ((size_t)i * emc::kAvgMaxSym + k) * 9;
        // row r of A * S (column-major product)
        for (int r = 0; r < 3; ++r)
          for (int cidx = 0; cidx < 3; ++cidx) {
            double v = 0.0;
            for (int q = 0; q < 3; ++q) v += A[r + 3 * q] * S[q + 3 * cidx];
            m[3 * r + cidx] = (float)v;
          }
      }
      emc::AvgParticle& pr = parts[i];
      for (int d = 0; d < 3; ++d) pr.shift[d] = shift ? shift[3 * (size_t)p + d] : 0.f;
      pr.weight = weight ? weight[p] : 1.f;
      pr.half = half[p];
      pr.wedge = a->nw ? wedge_index[p] : -1;
      pr.nsym = a->nsym;
      pr.pad = 0;
      widx[i] = pr.wedge;
    }
    // the batch's launches; on a failure the stream is drained before returning, since kernels
    // already queued may still read the mapped staging that the next call overwrites
    auto launch_batch = [&]() -> emc_status {
      emc::k_avg_stage_in<<<64, 256, 0, st>>>(d_mats_h, d_parts_h, d_widx_h, nb, a->nsym, a->mats, a->parts,
                                               a->widx);
      EMC_LAUNCH_CHECK();
      EMC_CUDA(cudaMemsetAsync(a->stats, 0, sizeof(emc::AvgStats) * nb, st));
      const int bricks = ((a->n + emc::kBrick - 1) / emc::kBrick) * ((a->n + emc::kBrick - 1) / emc::kBrick) *
                         ((a->n + emc::kBrick - 1) / emc::kBrick);
      emc::k_avg_rotate<<<dim3(bricks, nb), 256, 0, st>>>(d_particles + (size_t)b0 * a->nv, a->nv, nullptr, a->n,
                                                                a->mats, a->parts, 1, a->mask, a->bin_thr, a->rot,
                                                                a->stats);
      EMC_LAUNCH_CHECK();
      if (a->nw) {
        const int wb = ((a->nw + emc::kBrick - 1) / emc::kBrick) * ((a->nw + emc::kBrick - 1) / emc::kBrick) *
                       ((a->nw + emc::kBrick - 1) / emc::kBrick);
        emc::k_avg_rotate<<<dim3(wb, nb), 256, 0, st>>>(d_wedges, a->nvw, a->widx, a->nw, a->mats, a->parts, 0,
                                                              nullptr, 0.f, a->wrot, nullptr);
        EMC_LAUNCH_CHECK();
      }
      emc::k_avg_coef<<<(nb + 127) / 128, 128, 0, st>>>(a->stats, a->parts, nb, a->n_bin, a->mask_sum, (double)a->nv,
                                                       a->coef, a->counts, a->kept);
      EMC_LAUNCH_CHECK();
      const size_t smem = sizeof(float4) * nb;
      if (smem > 48 * 1024) EMC_CUDA(cudaFuncSetAttribute(emc::k_avg_accumulate,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      emc::k_avg_accumulate<<<grid_for(a->nv), 256, smem, st>>>(a->rot, a->nv, nb, a->coef, a->parts, a->mask, 1,
                                                                a->sum[0], a->sum[1]);
      EMC_LAUNCH_CHECK();
      if (a->nw) {
        emc::k_avg_accumulate<<<grid_for(a->nvw), 256, smem, st>>>(a->wrot, a->nvw, nb, a->coef, a->parts, nullptr, 0,
                                                                   a->wsum[0], a->wsum[1]);
        EMC_LAUNCH_CHECK();
      }
      return EMC_OK;
    };
    const emc_status rs = launch_batch();
    if (rs != EMC_OK) {
      cudaStreamSynchronize(st);
      return rs;
    }
    if (kept) {
      EMC_CUDA(cudaMemcpyAsync(kept_h.data(), a->kept, sizeof(int) * nb, cudaMemcpyDeviceToHost, st));
      EMC_CUDA(cudaStreamSynchronize(st));
      std::copy(kept_h.begin(), kept_h.begin() + nb, kept + b0);
    } else {
      // the host staging vectors are reused by the next batch
      EMC_CUDA(cudaStreamSynchronize(st));
    }
  }
  return EMC_OK;
}

emc_status emc_average_result(emc_average_t a, int half, float* d_avg, float* d_wedge_sum, long* count,
                              void* stream) {
  EMC_CHECK_ARG(a, "emc_average_result: null handle");
  EMC_CHECK_ARG(half == 1 || half == 2, "emc_average_result: half set %d (must be 1 or 2)", half);
  EMC_CHECK_ARG(!d_wedge_sum || a->nw, "emc_average_result: the handle averages no wedges");
  cudaStream_t st = emc::as_stream(stream);
  unsigned long long c[2] = {0, 0};
  EMC_CUDA(cudaMemcpyAsync(c, a->counts, sizeof(c), cudaMemcpyDeviceToHost, st));
  EMC_CUDA(cudaStreamSynchronize(st));
  const unsigned long long nh = c[half - 1];
  if (count) *count = (long)nh;
  if (d_avg) {
    // sum / count; a half set with no particle gives 0 / 0 = NaN as in MATLAB
    if (nh) {
      emc::k_avg_finish<<<grid_for(a->nv), 256, 0, st>>>(a->sum[half - 1], a->nv, (float)nh, d_avg);
      EMC_LAUNCH_CHECK();
    } else {
      EMC_CUDA(cudaMemsetAsync(d_avg, 0xff, sizeof(float) * a->nv, st));  // NaN, as 0 / 0
    }
  }
  if (d_wedge_sum)
    EMC_CUDA(cudaMemcpyAsync(d_wedge_sum, a->wsum[half - 1], sizeof(float) * a->nvw, cudaMemcpyDeviceToDevice, st));
  return EMC_OK;
}

emc_status emc_average_boxes(emc_average_t a, int* n, int* nw) {
  EMC_CHECK_ARG(a && n && nw, "emc_average_boxes: null argument");
  *n = a->n;
  *nw = a->nw;
  return EMC_OK;
}

emc_status emc_average_destroy(emc_average_t a) {
  if (!a) return EMC_OK;
  avg_free(a);
  delete a;
  return EMC_OK;
}

}  // extern "C"
