/*
 * mex.h -- the part of MATLAB's C matrix / MEX API that the gateways in this
 * directory use, declared from MATLAB's public documentation so that they
 * compile (and can be exercised by a stand-in runtime) where MATLAB is not
 * installed.  Inside MATLAB, `mex` puts its own mex.h first on the include
 * path and this file is not used.  Large-array-dims convention: mwSize and
 * mwIndex are size_t.
 */
#ifndef BN_MEX_SHIM_H
#define BN_MEX_SHIM_H

#include <stdbool.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;

typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum {
  mxUNKNOWN_CLASS = 0,
  mxCELL_CLASS,
  mxSTRUCT_CLASS,
  mxLOGICAL_CLASS,
  mxCHAR_CLASS,
  mxVOID_CLASS,
  mxDOUBLE_CLASS,
  mxSINGLE_CLASS,
  mxINT8_CLASS,
  mxUINT8_CLASS,
  mxINT16_CLASS,
  mxUINT16_CLASS,
  mxINT32_CLASS,
  mxUINT32_CLASS,
  mxINT64_CLASS,
  mxUINT64_CLASS
} mxClassID;

bool mxIsSparse(const mxArray* pa);
bool mxIsInt32(const mxArray* pa);
size_t mxGetM(const mxArray* pa);
size_t mxGetN(const mxArray* pa);
size_t mxGetNumberOfElements(const mxArray* pa);
mwIndex* mxGetJc(const mxArray* pa);
mwIndex* mxGetIr(const mxArray* pa);
double* mxGetPr(const mxArray* pa);
void* mxGetData(const mxArray* pa);
double mxGetScalar(const mxArray* pa);

mxArray* mxCreateSparse(mwSize m, mwSize n, mwSize nzmax, mxComplexity flag);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity flag);
mxArray* mxCreateDoubleScalar(double value);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);

void* mxMalloc(size_t n);
void* mxCalloc(size_t n, size_t size);
void mxFree(void* ptr);

/* does not return */
void mexErrMsgIdAndTxt(const char* errorid, const char* errormsg, ...);

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);

#ifdef __cplusplus
}
#endif
#endif /* BN_MEX_SHIM_H */
