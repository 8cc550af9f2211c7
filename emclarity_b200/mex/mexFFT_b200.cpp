// mexFFT gateway on libemc_b200 (reference: mexFiles/mexFFT.cu:16-239).
//   [ft, planF, planI] = mexFFT(gpuArray x, int16 invTrim)        first call makes the plan
//   ft                 = mexFFT(gpuArray x, invTrim, planF, planI) reuse
//                        mexFFT(scalar, invTrim, planF, planI)     free the plan
// Direction follows the complexity of x (real -> R2C, complex -> C2R), unnormalised like
// cufftExecR2C / cufftExecC2R.  Output x-size: n/2+1 forward, 2*nh - invTrim inverse.
#include "mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs < 2) mexErrMsgIdAndTxt("EMC:mexFFT:rhs", "expected at least 2 inputs");
  if (!mxGPUIsValidGPUData(prhs[0])) mexErrMsgIdAndTxt("EMC:mexFFT:rhs", "This inputArray is not valid gpudata.");
  const mxGPUArray* in = mxGPUCreateFromMxArray(prhs[0]);
  const int inv_trim = (int)mex_num(prhs[1]);
  emc_fft_t plan = nullptr;
  if (nrhs > 2) {
    plan = (emc_fft_t)(uintptr_t)mex_handle(prhs[2]);
    if (mxGPUGetNumberOfElements(in) == 1) {
      emc_fft_destroy(plan);
      mxGPUDestroyGPUArray(in);
      return;
    }
  }
  const mwSize nd = mxGPUGetNumberOfDimensions(in);
  const mwSize* d = mxGPUGetDimensions(in);
  const bool fwd = mxGPUGetComplexity(in) == mxREAL;
  mwSize out_dims[3] = {d[0], nd > 1 ? d[1] : 1, nd > 2 ? d[2] : 1};
  out_dims[0] = fwd ? d[0] / 2 + 1 : 2 * d[0] - inv_trim;
  const int n[3] = {(int)(fwd ? d[0] : out_dims[0]), (int)out_dims[1], (int)out_dims[2]};
  const int rank = n[2] > 1 ? 3 : (n[1] > 1 ? 2 : 1);
  const bool made = plan == nullptr;
  if (made) EMC_MEX_CHECK("mexFFT", emc_fft_plan(rank, n, 1, &plan));
  mxGPUArray* out = mxGPUCreateGPUArray(nd < 3 ? nd : 3, out_dims, mxSINGLE_CLASS, fwd ? mxCOMPLEX : mxREAL,
                                        MX_GPU_DO_NOT_INITIALIZE);
  if (fwd)
    EMC_MEX_CHECK("mexFFT", emc_fft_r2c(plan, (const float*)mxGPUGetDataReadOnly(in), (float*)mxGPUGetData(out),
                                        nullptr));
  else
    EMC_MEX_CHECK("mexFFT", emc_fft_c2r(plan, (const float*)mxGPUGetDataReadOnly(in), (float*)mxGPUGetData(out),
                                        nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(out);
  mxGPUDestroyGPUArray(out);
  mxGPUDestroyGPUArray(in);
  if (made) {
    if (nlhs > 1) plhs[1] = mex_new_handle((uint64_t)(uintptr_t)plan);
    else emc_fft_destroy(plan);
    if (nlhs > 2) plhs[2] = mex_new_handle(0);
  }
}
