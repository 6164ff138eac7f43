/* Declarations of the parts of MATLAB's documented C API (matrix.h / mex.h, interleaved complex, R2018a+)
 * that the MEX gateway mex/rtm_mex.c uses, so that tests/test_c_consumer.py can compile the gateway
 * for a syntax and type check where MATLAB is not installed. A stand-in for checking only: a real build
 * uses MATLAB's own mex.h through `mex -R2018a`. */
#ifndef RTM_TEST_MEX_STUB_H
#define RTM_TEST_MEX_STUB_H

#include <stdbool.h>
#include <stddef.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef double mxDouble;
typedef bool mxLogical;
typedef struct { mxDouble real, imag; } mxComplexDouble;
typedef enum { mxREAL, mxCOMPLEX } mxComplexity;
typedef enum { mxDOUBLE_CLASS = 6, mxUINT64_CLASS = 15 } mxClassID;

int mxGetString(const mxArray* a, char* buf, mwSize len);
double mxGetScalar(const mxArray* a);
bool mxIsEmpty(const mxArray* a);
bool mxIsComplex(const mxArray* a);
size_t mxGetM(const mxArray* a);
size_t mxGetN(const mxArray* a);
size_t mxGetNumberOfElements(const mxArray* a);
void* mxGetData(const mxArray* a);
mxDouble* mxGetDoubles(const mxArray* a);
mxComplexDouble* mxGetComplexDoubles(const mxArray* a);
mxArray* mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID id, mxComplexity c);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** names);
mxArray* mxCreateLogicalScalar(mxLogical v);
mxArray* mxCreateDoubleScalar(double v);
void mxSetField(mxArray* a, mwIndex i, const char* name, mxArray* v);
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...);

#endif
