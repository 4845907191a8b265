/* Minimal declarations of the MATLAB MEX API used by imogen_b200_mex.c, so that the gateway can be
 * compile-checked where MATLAB is not installed.  Declarations only: nothing here is called. */
#ifndef IMOGEN_TEST_MEX_STUB_H
#define IMOGEN_TEST_MEX_STUB_H
#include <stddef.h>
#include <stdio.h>
typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef enum { mxDOUBLE_CLASS = 6, mxUINT64_CLASS = 15 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
int mxGetString(const mxArray*, char*, mwSize);
double* mxGetPr(const mxArray*);
void* mxGetData(const mxArray*);
double mxGetScalar(const mxArray*);
size_t mxGetNumberOfElements(const mxArray*);
mwSize mxGetNumberOfDimensions(const mxArray*);
const mwSize* mxGetDimensions(const mxArray*);
int mxIsUint64(const mxArray*);
int mxIsDouble(const mxArray*);
int mxIsComplex(const mxArray*);
mxArray* mxCreateNumericMatrix(mwSize, mwSize, mxClassID, mxComplexity);
mxArray* mxCreateNumericArray(mwSize, const mwSize*, mxClassID, mxComplexity);
mxArray* mxCreateDoubleScalar(double);
mxArray* mxCreateString(const char*);
void mexErrMsgIdAndTxt(const char*, const char*, ...);
#endif
