// mexEmcSearch -- MEX gateway for the fused orientation search (no single reference MEX: it
// replaces the per-orientation MATLAB loop of alignment/BH_alignRaw3d_v2.m:1119-1423).
//   [cc, peak, best] = mexEmcSearch(gpuArray single ref, gpuArray single mask or [],
//                                   gpuArray single particle, gpuArray single wdgMask or [],
//                                   double prior[9], double eulers[n x 3], int peakRadius
//                                   [, gpuArray single refWdg or []])
//   wdgMask / refWdg: real half spectra ((n/2+1) x n x n, FFT order), the weights of
//   BH_multi_xcf_Translational_2.m:35-38 on the rotated reference (the particle's wedge) and on
//   the particle (the reference's wedge); [] = 1.
//   cc:   n x 1 single (normalised CC at each orientation's peak)
//   peak: n x 3 int32  (integer shift x, y, z)
//   best: 1 x 5 double [cc, orientation (1-based), dx, dy, dz]
#include <cuda_runtime.h>

#include <vector>

#include "mex_common.h"

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
  if (nrhs != 7 && nrhs != 8) mexErrMsgIdAndTxt("EMC:mexEmcSearch:rhs", "expected 7 or 8 inputs");
  const mxGPUArray* ref = mxGPUCreateFromMxArray(prhs[0]);
  const int n = (int)mxGPUGetDimensions(ref)[0];
  const float* mask = nullptr;
  const mxGPUArray* gm = nullptr;
  if (mxGetNumberOfElements(prhs[1]) > 0) {
    gm = mxGPUCreateFromMxArray(prhs[1]);
    mask = (const float*)mxGPUGetDataReadOnly(gm);
  }
  const mxGPUArray* part = mxGPUCreateFromMxArray(prhs[2]);
  const float* wdg_mask = nullptr;
  const mxGPUArray* gw = nullptr;
  if (mxGetNumberOfElements(prhs[3]) > 0) {
    gw = mxGPUCreateFromMxArray(prhs[3]);
    wdg_mask = (const float*)mxGPUGetDataReadOnly(gw);
  }
  const float* ref_wdg = nullptr;
  const mxGPUArray* grw = nullptr;
  if (nrhs == 8 && mxGetNumberOfElements(prhs[7]) > 0) {
    grw = mxGPUCreateFromMxArray(prhs[7]);
    ref_wdg = (const float*)mxGPUGetDataReadOnly(grw);
  }
  emc_particle_desc d;
  memset(&d, 0, sizeof(d));
  for (int i = 0; i < 9; ++i) d.prior[i] = mex_num(prhs[4], i);
  const int no = (int)(mxGetNumberOfElements(prhs[5]) / 3);
  std::vector<double> ptp(3 * (size_t)no);
  for (int o = 0; o < no; ++o)
    for (int k = 0; k < 3; ++k) ptp[3 * o + k] = mex_num(prhs[5], o + (size_t)k * no);  // n x 3 column-major
  const int radius = (int)mex_num(prhs[6]);
  const mwSize hd[3] = {(mwSize)(n / 2 + 1), (mwSize)n, (mwSize)n};
  mxGPUArray* spec = mxGPUCreateGPUArray(3, hd, mxSINGLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE);
  const mwSize one = 1;
  mxGPUArray* en = mxGPUCreateGPUArray(1, &one, mxDOUBLE_CLASS, mxREAL, MX_GPU_INITIALIZE_VALUES);
  EMC_MEX_CHECK("mexEmcSearch", emc_particle_spectrum(n, (const float*)mxGPUGetDataReadOnly(part), ref_wdg, nullptr,
                                                      (float*)mxGPUGetData(spec), (double*)mxGPUGetData(en),
                                                      nullptr));
  emc_search_t s = nullptr;
  EMC_MEX_CHECK("mexEmcSearch", emc_search_create(&s));
  int rid = -1;
  emc_status st = emc_search_add_reference(s, (const float*)mxGPUGetDataReadOnly(ref), n, mask, nullptr,
                                           EMC_DTYPE_F32, &rid, nullptr);
  if (st == EMC_OK) st = emc_search_set_orientations(s, ptp.data(), no);
  if (st == EMC_OK) st = emc_search_configure(s, radius, EMC_INTERP_LINEAR, 0);
  double e = 0;
  if (st == EMC_OK) st = cudaMemcpy(&e, mxGPUGetData(en), sizeof(double), cudaMemcpyDeviceToHost) ? EMC_E_CUDA : EMC_OK;
  std::vector<float> cc(no);
  std::vector<int> pk(3 * (size_t)no);
  emc_search_hit hit;
  if (st == EMC_OK) {
    d.spectrum = (const float*)mxGPUGetData(spec);
    d.energy = e;
    d.box = n;
    d.ref_id = rid;
    d.orient_begin = 0;
    d.orient_count = no;
    d.wedge = wdg_mask;
    st = emc_search_run_host(s, &d, 1, cc.data(), pk.data(), &hit, nullptr);
  }
  emc_search_destroy(s);
  mxGPUDestroyGPUArray(spec);
  mxGPUDestroyGPUArray(en);
  mxGPUDestroyGPUArray(ref);
  mxGPUDestroyGPUArray(part);
  if (gm) mxGPUDestroyGPUArray(gm);
  if (gw) mxGPUDestroyGPUArray(gw);
  if (grw) mxGPUDestroyGPUArray(grw);
  EMC_MEX_CHECK("mexEmcSearch", st);
  mwSize cd[2] = {(mwSize)no, 1};
  plhs[0] = mxCreateNumericArray(2, cd, mxSINGLE_CLASS, mxREAL);
  memcpy(mxGetData(plhs[0]), cc.data(), sizeof(float) * no);
  if (nlhs > 1) {
    mwSize pd[2] = {(mwSize)no, 3};
    plhs[1] = mxCreateNumericArray(2, pd, mxINT32_CLASS, mxREAL);
    int* p = (int*)mxGetData(plhs[1]);
    for (int o = 0; o < no; ++o)
      for (int k = 0; k < 3; ++k) p[o + (size_t)k * no] = pk[3 * o + k];
  }
  if (nlhs > 2) {
    mwSize bd[2] = {1, 5};
    plhs[2] = mxCreateNumericArray(2, bd, mxDOUBLE_CLASS, mxREAL);
    double* b = (double*)mxGetData(plhs[2]);
    b[0] = hit.cc; b[1] = hit.orient + 1; b[2] = hit.peak[0]; b[3] = hit.peak[1]; b[4] = hit.peak[2];
  }
}
