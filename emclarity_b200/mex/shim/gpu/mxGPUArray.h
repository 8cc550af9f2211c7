/* gpu/mxGPUArray.h -- gpuArray part of the minimal MEX stand-in (see mex.h). */
#ifndef EMC_MEX_SHIM_MXGPUARRAY_H
#define EMC_MEX_SHIM_MXGPUARRAY_H
#include "../matrix.h"

typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_DO_NOT_INITIALIZE = 0, MX_GPU_INITIALIZE_VALUES = 1 } mxGPUInitialize;

#ifdef __cplusplus
extern "C" {
#endif
int mxInitGPU(void);
int mxGPUIsValidGPUData(const mxArray* a);
const mxGPUArray* mxGPUCreateFromMxArray(const mxArray* a);
mxGPUArray* mxGPUCreateGPUArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx,
                                mxGPUInitialize init);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray* a);
const mwSize* mxGPUGetDimensions(const mxGPUArray* a);
mwSize mxGPUGetNumberOfElements(const mxGPUArray* a);
mxComplexity mxGPUGetComplexity(const mxGPUArray* a);
mxClassID mxGPUGetClassID(const mxGPUArray* a);
void* mxGPUGetData(mxGPUArray* a);
const void* mxGPUGetDataReadOnly(const mxGPUArray* a);
mxArray* mxGPUCreateMxArrayOnGPU(const mxGPUArray* a);
void mxGPUDestroyGPUArray(const mxGPUArray* a);
#ifdef __cplusplus
}
#endif
#endif
