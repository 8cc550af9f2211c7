// mexEmcAverage -- MEX gateway for the subtomogram averaging loop (no single reference MEX: it
// replaces the per-particle interpolator / normalise / accumulate body of
// transformations/BH_average3d.m:1417-1482 and the division of :1703-1707).
//   h = mexEmcAverage(gpuArray single mask, double sym[3 x 3 x k] or [], int32 wedgeBox, single binThr)
//   kept = mexEmcAverage(h, gpuArray single particles[n x n x n x p], double rot[9 x p],
//                        single shift[3 x p], single peakWgt[p], int32 half[p],
//                        gpuArray single wedges[nw x nw x nw x w] or [], int32 wedgeIndex[p] (1-based))
//   [avg, wedgeSum, count] = mexEmcAverage(h, int32 half)      (gpuArrays; wedgeSum [] without wedges)
//   mexEmcAverage(h)                                            (frees the handle)
#include <cuda_runtime.h>

#include <vector>

#include "mex_common.h"

static void do_create(int nlhs, mxArray* plhs[], const mxArray* prhs[]) {
  const mxGPUArray* gm = mxGPUCreateFromMxArray(prhs[0]);
  const int n = (int)mxGPUGetDimensions(gm)[0];
  const size_t ns = mxGetNumberOfElements(prhs[1]) / 9;
  std::vector<double> sym(9 * ns);
  for (size_t i = 0; i < 9 * ns; ++i) sym[i] = mex_num(prhs[1], i);
  const int nw = (int)mex_num(prhs[2]);
  const float thr = (float)mex_num(prhs[3]);
  emc_average_t a = nullptr;
  const emc_status st = emc_average_create(n, (const float*)mxGPUGetDataReadOnly(gm), thr, nw,
                                           ns ? sym.data() : nullptr, ns ? (int)ns : 1, 0, &a, nullptr);
  mxGPUDestroyGPUArray(gm);
  EMC_MEX_CHECK("mexEmcAverage", st);
  (void)nlhs;
  plhs[0] = mex_new_handle((uint64_t)(uintptr_t)a);
}

static void do_add(int nlhs, mxArray* plhs[], const mxArray* prhs[]) {
  emc_average_t a = (emc_average_t)(uintptr_t)mex_handle(prhs[0]);
  const mxGPUArray* gp = mxGPUCreateFromMxArray(prhs[1]);
  const size_t count = mxGetNumberOfElements(prhs[5]);
  std::vector<double> rot(9 * count);
  std::vector<float> shift(3 * count), weight(count);
  std::vector<int> half(count), widx(count), kept(count);
  for (size_t i = 0; i < 9 * count; ++i) rot[i] = mex_num(prhs[2], i);
  for (size_t i = 0; i < 3 * count; ++i) shift[i] = (float)mex_num(prhs[3], i);
  for (size_t i = 0; i < count; ++i) {
    weight[i] = (float)mex_num(prhs[4], i);
    half[i] = (int)mex_num(prhs[5], i);
  }
  const mxGPUArray* gw = nullptr;
  const float* wedges = nullptr;
  int n_wedges = 0;
  if (mxGetNumberOfElements(prhs[6]) > 0) {
    gw = mxGPUCreateFromMxArray(prhs[6]);
    wedges = (const float*)mxGPUGetDataReadOnly(gw);
    const mwSize nd = mxGPUGetNumberOfDimensions(gw);
    n_wedges = nd > 3 ? (int)mxGPUGetDimensions(gw)[3] : 1;
    for (size_t i = 0; i < count; ++i) widx[i] = (int)mex_num(prhs[7], i) - 1;
  }
  const emc_status st = emc_average_add(a, (const float*)mxGPUGetDataReadOnly(gp), (int)count, rot.data(),
                                        shift.data(), weight.data(), half.data(), wedges, n_wedges,
                                        gw ? widx.data() : nullptr, kept.data(), nullptr);
  mxGPUDestroyGPUArray(gp);
  if (gw) mxGPUDestroyGPUArray(gw);
  EMC_MEX_CHECK("mexEmcAverage", st);
  (void)nlhs;
  mwSize d[2] = {(mwSize)count, 1};
  plhs[0] = mxCreateNumericArray(2, d, mxINT32_CLASS, mxREAL);
  memcpy(mxGetData(plhs[0]), kept.data(), sizeof(int) * count);
}

static void do_result(int nlhs, mxArray* plhs[], const mxArray* prhs[]) {
  emc_average_t a = (emc_average_t)(uintptr_t)mex_handle(prhs[0]);
  const int half = (int)mex_num(prhs[1]);
  // box sizes: query the count first (validates the handle and the half set)
  long count = 0;
  EMC_MEX_CHECK("mexEmcAverage", emc_average_result(a, half, nullptr, nullptr, &count, nullptr));
  int n = 0, nw = 0;
  EMC_MEX_CHECK("mexEmcAverage", emc_average_boxes(a, &n, &nw));
  const mwSize dn[3] = {(mwSize)n, (mwSize)n, (mwSize)n};
  mxGPUArray* avg = mxGPUCreateGPUArray(3, dn, mxSINGLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
  mxGPUArray* ws = nullptr;
  if (nw) {
    const mwSize dw[3] = {(mwSize)nw, (mwSize)nw, (mwSize)nw};
    ws = mxGPUCreateGPUArray(3, dw, mxSINGLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
  }
  const emc_status st = emc_average_result(a, half, (float*)mxGPUGetData(avg), ws ? (float*)mxGPUGetData(ws) : nullptr,
                                           &count, nullptr);
  if (st == EMC_OK) cudaDeviceSynchronize();
  plhs[0] = mxGPUCreateMxArrayOnGPU(avg);
  mxGPUDestroyGPUArray(avg);
  if (nlhs > 1) {
    if (ws) {
      plhs[1] = mxGPUCreateMxArrayOnGPU(ws);
    } else {
      mwSize z[2] = {0, 0};
      plhs[1] = mxCreateNumericArray(2, z, mxSINGLE_CLASS, mxREAL);
    }
  }
  if (ws) mxGPUDestroyGPUArray(ws);
  if (nlhs > 2) {
    mwSize one[2] = {1, 1};
    plhs[2] = mxCreateNumericArray(2, one, mxDOUBLE_CLASS, mxREAL);
    *(double*)mxGetData(plhs[2]) = (double)count;
  }
  EMC_MEX_CHECK("mexEmcAverage", st);
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  switch (nrhs) {
    case 4: do_create(nlhs, plhs, prhs); break;
    case 8: do_add(nlhs, plhs, prhs); break;
    case 2: do_result(nlhs, plhs, prhs); break;
    case 1: emc_average_destroy((emc_average_t)(uintptr_t)mex_handle(prhs[0])); break;
    default: mexErrMsgIdAndTxt("EMC:mexEmcAverage:rhs", "expected 4 (create), 8 (add), 2 (result) or 1 (free) inputs");
  }
}
