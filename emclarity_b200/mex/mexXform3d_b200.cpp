// mexXform3d gateway on libemc_b200 (reference: mexFiles/mexXform3d.cu:93-324).
//   [out, h, dummy] = mexXform3d(uint64 size[3], gpuArray single vol, single R[9], single shift[3], logical fwd)
//   out             = mexXform3d(uint64 size[3], dummy, R, shift, fwd, uint64 h)    reuse the handle
//                     mexXform3d(uint64 h, dummy)                                   free the handle
// The handle replaces the reference's (texture object, cudaArray) pair; the second output is 0.
// Interpolation: trilinear with a zero-valued border, the reference texture's addressing mode.
#include "mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs == 2) {
    EMC_MEX_CHECK("mexXform3d", emc_xform3d_destroy((emc_volume_t)(uintptr_t)mex_handle(prhs[0])));
    return;
  }
  if (nrhs < 5) mexErrMsgIdAndTxt("EMC:mexXform3d:rhs", "expected 5 or 6 inputs");
  if (!mxGPUIsValidGPUData(prhs[1])) mexErrMsgIdAndTxt("EMC:mexXform3d:rhs", "Expected a 3d gpuarray.");
  const uint64_t* size = (const uint64_t*)mxGetData(prhs[0]);
  const int nx = (int)size[0], ny = (int)size[1], nz = (int)size[2];
  double R[9];
  for (int i = 0; i < 9; ++i) R[i] = mex_num(prhs[2], i);
  float sh[3];
  for (int i = 0; i < 3; ++i) sh[i] = (float)mex_num(prhs[3], i);
  const int fwd = mex_num(prhs[4]) != 0.0;
  emc_volume_t h = nullptr;
  bool created = false;
  if (nrhs > 5) {
    h = (emc_volume_t)(uintptr_t)mex_handle(prhs[5]);
  } else {
    const mxGPUArray* in = mxGPUCreateFromMxArray(prhs[1]);
    EMC_MEX_CHECK("mexXform3d", emc_xform3d_create((const float*)mxGPUGetDataReadOnly(in), nx, ny, nz,
                                                   EMC_DTYPE_F32, &h, nullptr));
    mxGPUDestroyGPUArray(in);
    created = true;
  }
  const mwSize dims[3] = {(mwSize)nx, (mwSize)ny, (mwSize)nz};
  mxGPUArray* out = mxGPUCreateGPUArray(3, dims, mxSINGLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
  EMC_MEX_CHECK("mexXform3d", emc_xform3d_apply(h, R, 1, sh, fwd, EMC_INTERP_LINEAR_BORDER,
                                                (float*)mxGPUGetData(out), nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(out);
  mxGPUDestroyGPUArray(out);
  if (created) {
    if (nlhs > 1) plhs[1] = mex_new_handle((uint64_t)(uintptr_t)h);
    else emc_xform3d_destroy(h);
    if (nlhs > 2) plhs[2] = mex_new_handle(0);
  }
}
