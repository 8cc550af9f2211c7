// mex_shim.cpp -- implementation of the minimal MEX / mxGPUArray stand-in.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <stdexcept>
#include <string>

#include "gpu/mxGPUArray.h"
#include "mex.h"

struct mxArray_tag {
  mxClassID cls;
  mxComplexity cplx;
  mwSize ndim;
  mwSize dims[8];
  void* data;
  bool gpu;
  bool owns;
};

struct mxGPUArray_tag {
  mxArray a;
};

static thread_local std::string g_err;

static size_t class_bytes(mxClassID c) {
  switch (c) {
    case mxLOGICAL_CLASS: case mxINT8_CLASS: case mxUINT8_CLASS: case mxCHAR_CLASS: return 1;
    case mxINT16_CLASS: case mxUINT16_CLASS: return 2;
    case mxSINGLE_CLASS: case mxINT32_CLASS: case mxUINT32_CLASS: return 4;
    default: return 8;
  }
}

static mwSize numel(const mxArray* a) {
  mwSize n = 1;
  for (mwSize i = 0; i < a->ndim; ++i) n *= a->dims[i];
  return n;
}

static size_t nbytes(const mxArray* a) { return numel(a) * class_bytes(a->cls) * (a->cplx == mxCOMPLEX ? 2 : 1); }

static void set_dims(mxArray* a, mwSize ndim, const mwSize* dims) {
  a->ndim = ndim < 2 ? 2 : ndim;
  for (mwSize i = 0; i < 8; ++i) a->dims[i] = 1;
  for (mwSize i = 0; i < ndim && i < 8; ++i) a->dims[i] = dims[i];
  // MATLAB drops trailing singleton dimensions beyond the second
  while (a->ndim > 2 && a->dims[a->ndim - 1] == 1) --a->ndim;
}

extern "C" {

void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = std::string(id ? id : "") + ": " + buf;
  throw std::runtime_error(g_err);
}

int mexPrintf(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int r = vfprintf(stderr, fmt, ap);
  va_end(ap);
  return r;
}

void mexMakeArrayPersistent(mxArray*) {}

const char* emc_shim_last_error(void) { return g_err.c_str(); }

void* mxGetData(const mxArray* a) { return a ? a->data : nullptr; }

mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
  mxArray* a = new mxArray_tag();
  a->cls = cls;
  a->cplx = cplx;
  set_dims(a, ndim, dims);
  a->gpu = false;
  a->owns = true;
  a->data = calloc(nbytes(a) ? nbytes(a) : 1, 1);
  return a;
}

void mxDestroyArray(mxArray* a) {
  if (!a) return;
  if (a->owns) {
    if (a->gpu) cudaFree(a->data);
    else free(a->data);
  }
  delete a;
}

mwSize mxGetNumberOfElements(const mxArray* a) { return numel(a); }
mxClassID mxGetClassID(const mxArray* a) { return a->cls; }
bool mxIsComplex(const mxArray* a) { return a->cplx == mxCOMPLEX; }

mxArray* emc_shim_wrap_host(void* data, mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
  mxArray* a = new mxArray_tag();
  a->cls = cls;
  a->cplx = cplx;
  set_dims(a, ndim, dims);
  a->data = data;
  a->gpu = false;
  a->owns = false;
  return a;
}

mxArray* emc_shim_wrap_gpu(void* data, mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
  mxArray* a = emc_shim_wrap_host(data, ndim, dims, cls, cplx);
  a->gpu = true;
  return a;
}

bool emc_shim_is_gpu(const mxArray* a) { return a->gpu; }

const mwSize* emc_shim_dims(const mxArray* a, mwSize* ndim) {
  *ndim = a->ndim;
  return a->dims;
}

int mxInitGPU(void) { return cudaFree(0) == cudaSuccess ? 0 : 1; }
int mxGPUIsValidGPUData(const mxArray* a) { return a && a->gpu; }

const mxGPUArray* mxGPUCreateFromMxArray(const mxArray* a) {
  mxGPUArray* g = new mxGPUArray_tag();
  g->a = *a;
  g->a.owns = false;
  return g;
}

mxGPUArray* mxGPUCreateGPUArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx,
                                mxGPUInitialize init) {
  mxGPUArray* g = new mxGPUArray_tag();
  g->a.cls = cls;
  g->a.cplx = cplx;
  set_dims(&g->a, ndim, dims);
  g->a.gpu = true;
  g->a.owns = true;
  size_t b = nbytes(&g->a);
  if (cudaMalloc(&g->a.data, b ? b : 1) != cudaSuccess) mexErrMsgIdAndTxt("shim:oom", "cudaMalloc(%zu)", b);
  if (init == MX_GPU_INITIALIZE_VALUES) cudaMemset(g->a.data, 0, b);
  return g;
}

mwSize mxGPUGetNumberOfDimensions(const mxGPUArray* g) { return g->a.ndim; }
const mwSize* mxGPUGetDimensions(const mxGPUArray* g) { return g->a.dims; }
mwSize mxGPUGetNumberOfElements(const mxGPUArray* g) { return numel(&g->a); }
mxComplexity mxGPUGetComplexity(const mxGPUArray* g) { return g->a.cplx; }
mxClassID mxGPUGetClassID(const mxGPUArray* g) { return g->a.cls; }
void* mxGPUGetData(mxGPUArray* g) { return g->a.data; }
const void* mxGPUGetDataReadOnly(const mxGPUArray* g) { return g->a.data; }

mxArray* mxGPUCreateMxArrayOnGPU(const mxGPUArray* g) {
  // the new mxArray takes over the device buffer
  mxArray* a = new mxArray_tag();
  *a = g->a;
  const_cast<mxGPUArray*>(g)->a.owns = false;
  return a;
}

void mxGPUDestroyGPUArray(const mxGPUArray* g) {
  if (!g) return;
  if (g->a.owns) cudaFree(g->a.data);
  delete g;
}

}  // extern "C"

// Calls the gateway's mexFunction, turning a mexErrMsgIdAndTxt into a return code of 1.
extern "C" int emc_shim_call(int nlhs, mxArray** plhs, int nrhs, const mxArray** prhs) {
  try {
    g_err.clear();
    mexFunction(nlhs, plhs, nrhs, prhs);
    return 0;
  } catch (const std::exception& e) {
    if (g_err.empty()) g_err = e.what();
    return 1;
  }
}
