// mexCTF gateway on libemc_b200 (reference: mexFiles/mexCTF.cu:6-121).
//   ctf = mexCTF(half, sq, nX, nY, pix, lambda, Cs, df1, df2, ast, AC[, centred[, occ, exposure]])
// Scalars may be of any numeric class (the reference reads nX / nY through an int pointer).
#include "mex_common.h"

void mexFunction(int, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 11 && nrhs != 12 && nrhs != 14) mexErrMsgIdAndTxt("EMC:mexCTF:rhs", "expected 11, 12 or 14 inputs");
  const int half = mex_num(prhs[0]) != 0.0, sq = mex_num(prhs[1]) != 0.0;
  const int nx = (int)mex_num(prhs[2]), ny = (int)mex_num(prhs[3]);
  emc_ctf_params p;
  p.pixel_size = (float)mex_num(prhs[4]);
  p.wavelength = (float)mex_num(prhs[5]);
  p.cs_mm = (float)mex_num(prhs[6]);
  p.defocus1 = (float)mex_num(prhs[7]);
  p.defocus2 = (float)mex_num(prhs[8]);
  p.astig_deg = (float)mex_num(prhs[9]);
  p.amp_contrast = (float)mex_num(prhs[10]);
  const int centred = nrhs >= 12 ? mex_num(prhs[11]) != 0.0 : 0;
  const mwSize dims[2] = {(mwSize)(half ? nx / 2 + 1 : nx), (mwSize)ny};
  mxGPUArray* out = mxGPUCreateGPUArray(2, dims, mxSINGLE_CLASS, mxREAL, MX_GPU_DO_NOT_INITIALIZE);
  // the reference gateway ignores occupancy / exposure (its weighted launch is commented out)
  EMC_MEX_CHECK("mexCTF", emc_ctf2d(&p, nx, ny, half, sq, centred, (float*)mxGPUGetData(out), nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(out);
  mxGPUDestroyGPUArray(out);
}
