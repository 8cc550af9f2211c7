// mex_common.h -- helpers shared by the MEX gateways of libemc_b200.
//
// The gateways keep the reference MEX names and argument orders (mexFiles/mexXform3d.cu:93,
// mexFFT.cu:16, mexCTF.cu:6, mexSF3D.cu:84) and forward to the C-ABI.  A non-zero status is
// turned into mexErrMsgIdAndTxt("EMC:<function>:<status>", ...).
#pragma once
#include <stdint.h>
#include <string.h>

#include "emc_b200.h"
#include "gpu/mxGPUArray.h"
#include "mex.h"

#define EMC_MEX_CHECK(fn, call)                                                                         \
  do {                                                                                                  \
    emc_status _s = (call);                                                                             \
    if (_s != EMC_OK) mexErrMsgIdAndTxt("EMC:" fn ":status", "%s (%s)", emc_status_string(_s), emc_last_error()); \
  } while (0)

// Numeric scalar or element i of any real numeric class, converted to double.
static inline double mex_num(const mxArray* a, size_t i = 0) {
  const void* p = mxGetData(a);
  switch (mxGetClassID(a)) {
    case mxDOUBLE_CLASS: return ((const double*)p)[i];
    case mxSINGLE_CLASS: return ((const float*)p)[i];
    case mxINT8_CLASS: return ((const int8_t*)p)[i];
    case mxUINT8_CLASS: return ((const uint8_t*)p)[i];
    case mxLOGICAL_CLASS: return ((const uint8_t*)p)[i];
    case mxINT16_CLASS: return ((const int16_t*)p)[i];
    case mxUINT16_CLASS: return ((const uint16_t*)p)[i];
    case mxINT32_CLASS: return ((const int32_t*)p)[i];
    case mxUINT32_CLASS: return ((const uint32_t*)p)[i];
    case mxINT64_CLASS: return (double)((const int64_t*)p)[i];
    case mxUINT64_CLASS: return (double)((const uint64_t*)p)[i];
    default: mexErrMsgIdAndTxt("EMC:mex:class", "unsupported numeric class"); return 0;
  }
}

static inline uint64_t mex_handle(const mxArray* a) { return *(const uint64_t*)mxGetData(a); }

static inline mxArray* mex_new_handle(uint64_t h) {
  mwSize one = 1;
  mxArray* a = mxCreateNumericArray(1, &one, mxUINT64_CLASS, mxREAL);
  *(uint64_t*)mxGetData(a) = h;
  return a;
}
