// xform3d.cu -- rotate + shift + interpolate a volume (mexXform3d replacement).
//
// Reference: mexFiles/mexXform3d.cu:22-87 (kernel), :93-324 (gateway: texture object built
// on first call, reused through the 6th argument, destroyed with nrhs == 2) and the
// interpolator class (testScripts/interpolator.m:29-154) that sums symmetry copies and
// divides by their number.  Here the handle keeps a plain device copy of the source (FP32
// or BF16) and the gather runs through the read-only data cache with FP32 weights.
#include <algorithm>
#include <new>

#include "interp.cuh"

namespace emc {

constexpr int kMaxSym = 60;

struct XformArgs {
  float m[kMaxSym][9];  // row-major rows of each sampling matrix (rm_1, rm_2, rm_3)
  int nsym;
  float shift[3];
  int fwd;
  int mode;
  int nx, ny, nz;
};

template <typename T>
__global__ void __launch_bounds__(256) k_xform3d(const T* __restrict__ src, float* __restrict__ out,
                                                 const XformArgs a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= a.nx || y >= a.ny) return;
  const int cx = a.nx / 2, cy = a.ny / 2, cz = a.nz / 2;
  float u = (float)(x - cx), v = (float)(y - cy), w = (float)(z - cz);
  if (a.fwd) { u -= a.shift[0]; v -= a.shift[1]; w -= a.shift[2]; }
  float acc = 0.f;
  for (int s = 0; s < a.nsym; ++s) {
    const float* m = a.m[s];
    float sx = fmaf(m[0], u, fmaf(m[1], v, m[2] * w));
    float sy = fmaf(m[3], u, fmaf(m[4], v, m[5] * w));
    float sz = fmaf(m[6], u, fmaf(m[7], v, m[8] * w));
    if (!a.fwd) { sx += a.shift[0]; sy += a.shift[1]; sz += a.shift[2]; }
    acc += sample(a.mode, src, a.nx, a.ny, a.nz, sx + (float)cx, sy + (float)cy, sz + (float)cz);
  }
  out[((long)z * a.ny + y) * a.nx + x] = a.nsym > 1 ? acc / (float)a.nsym : acc;
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

emc_status to_bf16(const float* in, __nv_bfloat16* out, long n, cudaStream_t st) {
  const int blocks = (int)std::min<long>((n + 255) / 256, 4L * device_sm_count());
  k_f32_to_bf16<<<blocks, 256, 0, st>>>(in, out, n);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

}  // namespace emc

struct emc_volume_s {
  int nx, ny, nz;
  int dtype;
  void* data;
};

extern "C" {

emc_status emc_xform3d_create(const float* d_src, int nx, int ny, int nz, int store_dtype, emc_volume_t* out,
                              void* stream) {
  EMC_CHECK_ARG(out && d_src, "emc_xform3d_create: null argument");
  *out = nullptr;
  EMC_CHECK_ARG(nx > 0 && ny > 0 && nz > 0, "emc_xform3d_create: bad size %d %d %d", nx, ny, nz);
  EMC_CHECK_ARG(store_dtype == EMC_DTYPE_F32 || store_dtype == EMC_DTYPE_BF16, "emc_xform3d_create: bad dtype");
  emc_volume_s* h = new (std::nothrow) emc_volume_s();
  EMC_CHECK_ARG(h, "emc_xform3d_create: host allocation failed");
  h->nx = nx; h->ny = ny; h->nz = nz; h->dtype = store_dtype;
  const long n = (long)nx * ny * nz;
  const size_t bytes = n * (store_dtype == EMC_DTYPE_F32 ? 4 : 2);
  cudaStream_t st = emc::as_stream(stream);
  if (cudaMalloc(&h->data, bytes) != cudaSuccess) {
    delete h;
    emc::set_error("emc_xform3d_create: cudaMalloc(%zu) failed", bytes);
    return EMC_E_OOM;
  }
  emc_status s = EMC_OK;
  if (store_dtype == EMC_DTYPE_F32) {
    if (cudaMemcpyAsync(h->data, d_src, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
      emc::set_error("emc_xform3d_create: copy failed");
      s = EMC_E_CUDA;
    }
  } else {
    s = emc::to_bf16(d_src, (__nv_bfloat16*)h->data, n, st);
  }
  if (s != EMC_OK) {
    cudaFree(h->data);
    delete h;
    return s;
  }
  *out = h;
  return EMC_OK;
}

emc_status emc_xform3d_apply(emc_volume_t h, const double* R, int nsym, const float shift[3], int fwd, int interp,
                             float* d_out, void* stream) {
  EMC_CHECK_ARG(h && R && d_out, "emc_xform3d_apply: null argument");
  EMC_CHECK_ARG(nsym >= 1 && nsym <= emc::kMaxSym, "emc_xform3d_apply: nsym %d not in 1..%d", nsym, emc::kMaxSym);
  EMC_CHECK_ARG(interp >= 0 && interp <= 2, "emc_xform3d_apply: interp %d", interp);
  emc::XformArgs a;
  for (int s = 0; s < nsym; ++s)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) a.m[s][3 * i + j] = (float)R[9 * s + i + 3 * j];  // row i of column-major R
  a.nsym = nsym;
  for (int i = 0; i < 3; ++i) a.shift[i] = shift ? shift[i] : 0.f;
  a.fwd = fwd ? 1 : 0;
  a.mode = interp;
  a.nx = h->nx; a.ny = h->ny; a.nz = h->nz;
  dim3 block(32, 8);
  dim3 grid((h->nx + 31) / 32, (h->ny + 7) / 8, h->nz);
  cudaStream_t st = emc::as_stream(stream);
  if (h->dtype == EMC_DTYPE_F32)
    emc::k_xform3d<float><<<grid, block, 0, st>>>((const float*)h->data, d_out, a);
  else
    emc::k_xform3d<__nv_bfloat16><<<grid, block, 0, st>>>((const __nv_bfloat16*)h->data, d_out, a);
  EMC_LAUNCH_CHECK();
  return EMC_OK;
}

emc_status emc_xform3d_destroy(emc_volume_t h) {
  if (!h) return EMC_OK;
  cudaFree(h->data);
  delete h;
  return EMC_OK;
}

}  // extern "C"
