/* matrix.h -- mxArray part of the minimal MEX stand-in (see mex.h). */
#ifndef EMC_MEX_SHIM_MATRIX_H
#define EMC_MEX_SHIM_MATRIX_H
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag mxArray;

#ifdef __cplusplus
extern "C" {
#endif
void* mxGetData(const mxArray* a);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
void mxDestroyArray(mxArray* a);
mwSize mxGetNumberOfElements(const mxArray* a);
mxClassID mxGetClassID(const mxArray* a);
bool mxIsComplex(const mxArray* a);
/* stand-in only: wrap existing host / device memory (not owned) */
mxArray* emc_shim_wrap_host(void* data, mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
mxArray* emc_shim_wrap_gpu(void* data, mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
bool emc_shim_is_gpu(const mxArray* a);
const mwSize* emc_shim_dims(const mxArray* a, mwSize* ndim);
const char* emc_shim_last_error(void);
#ifdef __cplusplus
}
#endif
#endif
