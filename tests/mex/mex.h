/* Declarations of the part of MATLAB's MEX / matrix API that
 * fcwt_b200/mex/fcwtmex.cpp uses (R2018a interleaved-complex API), so the
 * gateway can be compiled and exercised without MATLAB. TEST
 * INFRASTRUCTURE: tests/mex/fake_mx.cpp implements them on the heap. */
#ifndef FCWT_TEST_MEX_H
#define FCWT_TEST_MEX_H
#include <stddef.h>
typedef size_t mwSize;
typedef struct mxArray_tag mxArray;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef enum { mxSINGLE_CLASS = 7, mxDOUBLE_CLASS = 6 } mxClassID;
typedef struct { float real, imag; } mxComplexSingle;
#ifdef __cplusplus
extern "C" {
#endif
bool mxIsSingle(const mxArray* a);
bool mxIsDouble(const mxArray* a);
bool mxIsComplex(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
double mxGetScalar(const mxArray* a);
float* mxGetSingles(const mxArray* a);
mxComplexSingle* mxGetComplexSingles(const mxArray* a);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx);
void* mxMalloc(size_t n);
void mxFree(void* p);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);
void mexWarnMsgIdAndTxt(const char* id, const char* fmt, ...);
int mexAtExit(void (*fn)(void));
void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]);
#ifdef __cplusplus
}
#endif
#endif
