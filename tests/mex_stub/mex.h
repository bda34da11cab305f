/*
 * A stand-in for MATLAB's mex.h with the part of the MEX API that ToTem's MEX shim uses
 * (waveCuda.cpp: mxGetPr, mxGetScalar, mxCreateNumericMatrix, mexErrMsgTxt), so that the shim
 * compiles unchanged outside MATLAB and can be called from tests.  An mxArray here is a plain
 * rows x cols block of caller-owned (wrapped) or stub-owned (created) memory.  mexErrMsgTxt
 * records the message and returns (MATLAB would unwind to the prompt; the shim returns right
 * after calling it).  The mex_stub_* functions are for the tests that drive the shim.
 */
#ifndef TOTEM_TEST_MEX_STUB_H
#define TOTEM_TEST_MEX_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxDOUBLE_CLASS = 6, mxUINT32_CLASS = 13 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

double *mxGetPr(const mxArray *a);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID cls, mxComplexity flag);
void mexErrMsgTxt(const char *msg);
/* the MEX entry point the shim defines (C linkage, as MATLAB's own mex.h declares it) */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

/* test side */
mxArray *mex_stub_wrap(void *data, mwSize m, mwSize n);
void *mex_stub_data(const mxArray *a);
mwSize mex_stub_rows(const mxArray *a);
mwSize mex_stub_cols(const mxArray *a);
void mex_stub_free(mxArray *a);
const char *mex_stub_last_error(void);
int mex_stub_error_count(void);

#ifdef __cplusplus
}
#endif

#endif
