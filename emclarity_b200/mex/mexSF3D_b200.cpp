// mexSF3D gateway on libemc_b200 (reference: mexFiles/mexSF3D.cu:84-302).
//   sf3d = mexSF3D(half, sq, uint32 size[3], pix[n], lambda[n], Cs[n], df1[n], df2[n], ast[n], AC[n],
//                  uint32 nTilts, tilt[n], exposure[n], occupancy[n][, int16 launch])
#include <vector>

#include "mex_common.h"

void mexFunction(int, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 14 && nrhs != 15) mexErrMsgIdAndTxt("EMC:mexSF3D:rhs", "requires 14 inputs.");
  const int half = mex_num(prhs[0]) != 0.0, sq = mex_num(prhs[1]) != 0.0;
  unsigned size[3];
  for (int i = 0; i < 3; ++i) size[i] = (unsigned)mex_num(prhs[2], i);
  const unsigned nt = (unsigned)mex_num(prhs[10]);
  std::vector<float> a[10];
  const int idx[10] = {3, 4, 5, 6, 7, 8, 9, 11, 12, 13};
  for (int k = 0; k < 10; ++k) {
    a[k].resize(nt);
    for (unsigned t = 0; t < nt; ++t) a[k][t] = (float)mex_num(prhs[idx[k]], t);
  }
  const mwSize dims[3] = {size[0], size[1], size[2]};
  mxGPUArray* out = mxGPUCreateGPUArray(3, dims, mxSINGLE_CLASS, mxREAL, MX_GPU_INITIALIZE_VALUES);
  EMC_MEX_CHECK("mexSF3D", emc_sf3d(half, sq, size, a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                                    a[5].data(), a[6].data(), nt, a[7].data(), a[8].data(), a[9].data(),
                                    (float*)mxGPUGetData(out), nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(out);
  mxGPUDestroyGPUArray(out);
}
