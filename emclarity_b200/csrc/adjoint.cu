// adjoint.cu -- forward + adjoint of the masked normalised CC with respect to the pose.
//
// For pose (phi, theta, psi, t) the reference is sampled with tricubic interpolation at
//   s(p) = M (p - c - t) + c,   M = (R_prior * D)',  D = defineMatrix([phi, theta, psi-phi], 'inv')
// (the 'forward' sampling of BH_alignRaw3d_v2.m:1287-1291), masked, and correlated at zero lag
// with the real-space particle template h = unnormalised inverse FFT of Q:
//   CC = A / sqrt(E_R E_P),  A = sum r h,  E_R = n^3 sum r^2 - (sum r)^2  (DC-free, Parseval).
// One pass over the voxels accumulates, in FP64, A, sum r, sum r^2 and for each pose parameter k
// the sums H_k = sum h G_k, R_k = sum r G_k, S_k = sum G_k with G_k = dr/dk; then
//   dCC/dk = H_k / sqrt(E_R E_P) - CC / E_R * (n^3 R_k - sum r * S_k).
// The Euler-angle derivatives of M are formed on the host in FP64.
#include <math.h>

#include <algorithm>
#include <vector>

#include "search_kernels.cuh"

namespace emc {

constexpr int kAdjSums = 21;  // A, S1, S2, then (H, R, S) x 6

struct AdjPose {
  float m[9];       // sampling matrix rows
  float dm[3][9];   // d m / d(phi, theta, psi) per degree
  float t[3];
};

struct AdjItem {
  const void* ref;      // n^3 reference (float or bf16)
  const void* cells;    // (n+1)^3 trilinear corner cells of the reference (same type) or null
  const float* mask;    // n^3 or null
  const float* h;       // n^3 real-space particle template
  int n;
  int dtype;
  int interp;           // EMC_INTERP_CUBIC or EMC_INTERP_LINEAR (through the cells)
  AdjPose pose;
};

// Tricubic (Catmull-Rom) value and gradient from the plain volume.
template <typename T>
struct CubicSampler {
  const T* ref;
  int n;
  __device__ __forceinline__ float operator()(float sx, float sy, float sz, float g[3]) const {
    return sample_cubic_grad(ref, n, n, n, sx, sy, sz, g);
  }
};

// Trilinear value and gradient (interpn semantics, zero outside [0, n-1]) from the corner cells.
template <typename T>
struct CellSampler {
  const CellT<T>* cells;
  int n;
  __device__ __forceinline__ float operator()(float sx, float sy, float sz, float g[3]) const {
    float f[3];
    bool ok;
    const long ci = cell_index<EMC_INTERP_LINEAR>(n, sx, sy, sz, f, &ok);
    float v[8];
    cell_values(load_cell(cells + ci), v);
    const float c00 = fmaf(f[0], v[1] - v[0], v[0]), c10 = fmaf(f[0], v[3] - v[2], v[2]);
    const float c01 = fmaf(f[0], v[5] - v[4], v[4]), c11 = fmaf(f[0], v[7] - v[6], v[6]);
    const float c0 = fmaf(f[1], c10 - c00, c00), c1 = fmaf(f[1], c11 - c01, c01);
    const float d0 = fmaf(f[1], (v[3] - v[2]) - (v[1] - v[0]), v[1] - v[0]);
    const float d1 = fmaf(f[1], (v[7] - v[6]) - (v[5] - v[4]), v[5] - v[4]);
    g[0] = ok ? fmaf(f[2], d1 - d0, d0) : 0.f;
    g[1] = ok ? fmaf(f[2], (c11 - c01) - (c10 - c00), c10 - c00) : 0.f;
    g[2] = ok ? c1 - c0 : 0.f;
    return ok ? fmaf(f[2], c1 - c0, c0) : 0.f;
  }
};

// Each warp takes whole (y, z) rows, its lanes x = lane + 32 k: the row's index arithmetic and the
// y / z parts of the sample point are formed once per row (the same FP32 operations as per voxel).
// Whether an item samples through the trilinear corner cells (else tricubic from the volume).
__host__ __device__ inline bool adj_uses_cells(const AdjItem& it) {
  return it.interp == EMC_INTERP_LINEAR && it.cells != nullptr;
}

template <typename S>
__device__ __forceinline__ void adj_accumulate(const S sampler, const float* __restrict__ mask,
                                               const float* __restrict__ h, int n, const AdjPose& sp,
                                               float acc[kAdjSums]) {
  const int c = n / 2;
  const int lane = threadIdx.x & 31;
  const int warps = (int)(gridDim.x * (blockDim.x >> 5));
  const float* m = sp.m;
  for (int row = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)); row < n * n; row += warps) {
    const int y = row % n, z = row / n;
    const float u1 = (float)(y - c) - sp.t[1], u2 = (float)(z - c) - sp.t[2];
    const float py = fmaf(m[1], u1, m[2] * u2), qy = fmaf(m[4], u1, m[5] * u2), ry = fmaf(m[7], u1, m[8] * u2);
    const long rbase = (long)row * n;
    for (int x = lane; x < n; x += 32) {
      const long i = rbase + x;
      const float u0 = (float)(x - c) - sp.t[0];
      const float sx = fmaf(m[0], u0, py) + (float)c;
      const float sy = fmaf(m[3], u0, qy) + (float)c;
      const float sz = fmaf(m[6], u0, ry) + (float)c;
      const float mk = mask ? __ldg(mask + i) : 1.f;
      if (mk == 0.f) continue;  // a zero mask voxel adds nothing to any of the sums
      float g[3];
      const float v = sampler(sx, sy, sz, g);
      const float r = mk * v;
      const float hv = __ldg(h + i);
      g[0] *= mk; g[1] *= mk; g[2] *= mk;
      acc[0] += r * hv;
      acc[1] += r;
      acc[2] += r * r;
      // angle derivatives: ds/dk = dm_k u
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float* d = sp.dm[k];
        const float gk = g[0] * fmaf(d[0], u0, fmaf(d[1], u1, d[2] * u2)) +
                         g[1] * fmaf(d[3], u0, fmaf(d[4], u1, d[5] * u2)) +
                         g[2] * fmaf(d[6], u0, fmaf(d[7], u1, d[8] * u2));
        acc[3 + 3 * k] += hv * gk;
        acc[4 + 3 * k] += r * gk;
        acc[5 + 3 * k] += gk;
      }
      // shift derivatives: ds/dt_j = -M[:, j]
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float gk = -(g[0] * m[j] + g[1] * m[3 + j] + g[2] * m[6 + j]);
        acc[12 + 3 * j] += hv * gk;
        acc[13 + 3 * j] += r * gk;
        acc[14 + 3 * j] += gk;
      }
    }
  }
}

// One block-row (blockIdx.y) per item; partial sums reduced in FP64 and added atomically.  One
// instantiation per (storage type, sampler): an item whose combination differs leaves at once, so
// each combination runs with the registers its own sampler needs (the tricubic sampler's gradient
// needs far more than the trilinear one's).
template <typename T, bool LIN>
__global__ void __launch_bounds__(256) k_cc_adjoint(const AdjItem* __restrict__ items, double* __restrict__ sums) {
  __shared__ AdjItem it;
  __shared__ double red[kAdjSums][8];
  const int item = blockIdx.y;
  if (threadIdx.x == 0) it = items[item];
  __syncthreads();
  constexpr int dtype = sizeof(T) == 4 ? EMC_DTYPE_F32 : EMC_DTYPE_BF16;
  if (it.dtype != dtype || adj_uses_cells(it) != LIN) return;  // the same for the whole CTA
  float acc[kAdjSums];
#pragma unroll
  for (int k = 0; k < kAdjSums; ++k) acc[k] = 0.f;
  if constexpr (LIN)
    adj_accumulate(CellSampler<T>{reinterpret_cast<const CellT<T>*>(it.cells), it.n}, it.mask, it.h, it.n, it.pose,
                   acc);
  else
    adj_accumulate(CubicSampler<T>{reinterpret_cast<const T*>(it.ref), it.n}, it.mask, it.h, it.n, it.pose, acc);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < kAdjSums; ++k) {
    double v = (double)acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < kAdjSums) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    atomicAdd(sums + (long)item * kAdjSums + threadIdx.x, t);
  }
}

// Rz / Rx and their derivatives (per radian), column-major 3x3 products in FP64.
static void mat_mul(const double* a, const double* b, double* c) {
  double t[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += a[i + 3 * k] * b[k + 3 * j];
      t[i + 3 * j] = s;
    }
  for (int i = 0; i < 9; ++i) c[i] = t[i];
}
static void rz(double a, double* r, bool d) {
  const double c = cos(a), s = sin(a);
  // [[c,-s,0],[s,c,0],[0,0,1]] and its derivative [[-s,-c,0],[c,-s,0],[0,0,0]]
  const double v[9] = {d ? -s : c, d ? c : s, 0, d ? -c : -s, d ? -s : c, 0, 0, 0, d ? 0.0 : 1.0};
  for (int i = 0; i < 9; ++i) r[i] = v[i];
}
static void rx(double a, double* r, bool d) {
  const double c = cos(a), s = sin(a);
  const double v[9] = {d ? 0.0 : 1.0, 0, 0, 0, d ? -s : c, d ? c : s, 0, d ? -c : -s, d ? -s : c};
  for (int i = 0; i < 9; ++i) r[i] = v[i];
}

// D = defineMatrix([phi, theta, psi - phi], 'inv') = Rz(phi) Rx(theta) Rz(psi - phi) and the
// derivatives of M = (prior D)' with respect to phi, theta, psi (per degree).
static void pose_matrices(const double prior[9], const double* pose, AdjPose* out) {
  const double k = M_PI / 180.0;
  const double a1 = pose[0] * k, a2 = pose[1] * k, a3 = (pose[2] - pose[0]) * k;
  double Z1[9], X2[9], Z3[9], dZ1[9], dX2[9], dZ3[9], t[9], D[9], dD[3][9];
  rz(a1, Z1, false); rz(a1, dZ1, true);
  rx(a2, X2, false); rx(a2, dX2, true);
  rz(a3, Z3, false); rz(a3, dZ3, true);
  mat_mul(Z1, X2, t); mat_mul(t, Z3, D);
  // d/dphi: dZ1 X2 Z3 - Z1 X2 dZ3   (a3 = psi - phi)
  double p1[9], p2[9];
  mat_mul(dZ1, X2, t); mat_mul(t, Z3, p1);
  mat_mul(Z1, X2, t); mat_mul(t, dZ3, p2);
  for (int i = 0; i < 9; ++i) dD[0][i] = p1[i] - p2[i];
  mat_mul(Z1, dX2, t); mat_mul(t, Z3, dD[1]);
  mat_mul(Z1, X2, t); mat_mul(t, dZ3, dD[2]);
  double R[9], dR[3][9];
  mat_mul(prior, D, R);
  for (int j = 0; j < 3; ++j) mat_mul(prior, dD[j], dR[j]);
  // sampling matrix rows m[3i + j] = M(i, j) = R(j, i)
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      out->m[3 * i + j] = (float)R[j + 3 * i];
      for (int q = 0; q < 3; ++q) out->dm[q][3 * i + j] = (float)(dR[q][j + 3 * i] * k);
    }
  for (int j = 0; j < 3; ++j) out->t[j] = (float)pose[3 + j];
}

}  // namespace emc

// Defined in search.cu: access to a registered reference.
emc_status emc_search_reference_info(emc_search_t s, int ref_id, const void** data, const void** cells,
                                     const float** mask, int* n, int* dtype);

extern "C" {

emc_status emc_cc_adjoint_batch(emc_search_t s, int n_items, const int* ref_ids, const float* const* d_h,
                                const double* energy_p, const double* priors, const double* poses, int interp,
                                double* h_cc, double* h_grad, void* stream) {
  EMC_CHECK_ARG(interp == EMC_INTERP_LINEAR || interp == EMC_INTERP_CUBIC, "emc_cc_adjoint_batch: interp %d", interp);
  EMC_CHECK_ARG(s && ref_ids && d_h && energy_p && priors && poses && h_cc && h_grad,
                "emc_cc_adjoint_batch: null argument");
  EMC_CHECK_ARG(n_items > 0 && n_items <= 65535, "emc_cc_adjoint_batch: n_items %d", n_items);
  std::vector<emc::AdjItem> items(n_items);
  int max_n = 0;
  for (int i = 0; i < n_items; ++i) {
    EMC_CHECK_ARG(d_h[i], "emc_cc_adjoint_batch: item %d has no template", i);
    EMC_CHECK_ARG(energy_p[i] > 0.0, "emc_cc_adjoint_batch: item %d energy must be > 0", i);
    const void* data = nullptr;
    const void* cells = nullptr;
    const float* mask = nullptr;
    int n = 0, dtype = 0;
    EMC_TRY(emc_search_reference_info(s, ref_ids[i], &data, &cells, &mask, &n, &dtype));
    items[i].ref = data;
    items[i].cells = cells;
    items[i].interp = interp;
    items[i].mask = mask;
    items[i].h = d_h[i];
    items[i].n = n;
    items[i].dtype = dtype;
    emc::pose_matrices(priors + 9 * (size_t)i, poses + 6 * (size_t)i, &items[i].pose);
    max_n = std::max(max_n, n);
  }
  cudaStream_t st = emc::as_stream(stream);
  const size_t item_bytes = sizeof(emc::AdjItem) * n_items;
  const size_t sum_bytes = sizeof(double) * emc::kAdjSums * n_items;
  char* buf = nullptr;
  EMC_CUDA(cudaMallocAsync(&buf, item_bytes + sum_bytes + 64, st));
  emc::AdjItem* d_items = reinterpret_cast<emc::AdjItem*>(buf);
  double* d_sums = reinterpret_cast<double*>(buf + ((item_bytes + 15) / 16) * 16);
  std::vector<double> sums((size_t)emc::kAdjSums * n_items);
  emc_status rs = EMC_OK;
  if (cudaMemcpyAsync(d_items, items.data(), item_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(d_sums, 0, sum_bytes, st) != cudaSuccess) {
    emc::set_error("emc_cc_adjoint_batch: upload failed");
    rs = EMC_E_CUDA;
  }
  if (rs == EMC_OK) {
    const long nv = (long)max_n * max_n * max_n;
    // enough blocks per item to fill the GPU twice over (three trilinear CTAs fit per SM) without
    // starving the reduction
    const long want = std::max<long>(1, (8L * emc::device_sm_count() + n_items - 1) / n_items);
    const int bx = (int)std::max<long>(1, std::min<long>((nv + 2047) / 2048, want));
    // one launch per (storage type, sampler) present among the items
    bool present[2][2] = {{false, false}, {false, false}};
    for (const auto& it : items) present[it.dtype == EMC_DTYPE_BF16 ? 1 : 0][emc::adj_uses_cells(it) ? 1 : 0] = true;
    const dim3 grid(bx, n_items);
    if (present[0][0]) emc::k_cc_adjoint<float, false><<<grid, 256, 0, st>>>(d_items, d_sums);
    if (present[0][1]) emc::k_cc_adjoint<float, true><<<grid, 256, 0, st>>>(d_items, d_sums);
    if (present[1][0]) emc::k_cc_adjoint<__nv_bfloat16, false><<<grid, 256, 0, st>>>(d_items, d_sums);
    if (present[1][1]) emc::k_cc_adjoint<__nv_bfloat16, true><<<grid, 256, 0, st>>>(d_items, d_sums);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(sums.data(), d_sums, sum_bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      emc::set_error("emc_cc_adjoint_batch: kernel or copy failed");
      rs = EMC_E_CUDA;
    }
  }
  cudaFreeAsync(buf, st);
  if (rs != EMC_OK) return rs;
  for (int i = 0; i < n_items; ++i) {
    const double n3 = (double)items[i].n * items[i].n * items[i].n;
    const double* q = &sums[(size_t)emc::kAdjSums * i];
    const double A = q[0], S1 = q[1], S2 = q[2];
    const double er = n3 * S2 - S1 * S1;
    if (!(er > 0.0)) {
      h_cc[i] = NAN;
      for (int k = 0; k < 6; ++k) h_grad[6 * i + k] = NAN;
      continue;
    }
    const double norm = 1.0 / sqrt(er * energy_p[i]);
    const double cc = A * norm;
    h_cc[i] = cc;
    for (int k = 0; k < 6; ++k) {
      const double H = q[3 + 3 * k], R = q[4 + 3 * k], S = q[5 + 3 * k];
      h_grad[6 * i + k] = H * norm - cc / er * (n3 * R - S1 * S);
    }
  }
  return EMC_OK;
}

emc_status emc_cc_adjoint(emc_search_t s, int ref_id, const float* d_h, double energy_p, const double prior[9],
                          const double* poses, int n_poses, double* h_cc, double* h_grad, void* stream) {
  EMC_CHECK_ARG(s && d_h && prior && poses && h_cc && h_grad, "emc_cc_adjoint: null argument");
  EMC_CHECK_ARG(n_poses > 0 && n_poses <= 65535, "emc_cc_adjoint: n_poses %d", n_poses);
  std::vector<int> ids(n_poses, ref_id);
  std::vector<const float*> hs(n_poses, d_h);
  std::vector<double> en(n_poses, energy_p), pr(9 * (size_t)n_poses);
  for (int i = 0; i < n_poses; ++i)
    for (int k = 0; k < 9; ++k) pr[9 * (size_t)i + k] = prior[k];
  return emc_cc_adjoint_batch(s, n_poses, ids.data(), hs.data(), en.data(), pr.data(), poses, EMC_INTERP_CUBIC, h_cc,
                              h_grad, stream);
}

}  // extern "C"
