/* A minimal stand-in for MATLAB's mex.h: the declarations the MEX shim
 * uses, so its source can be compiled (syntax and types) where MATLAB is not
 * installed.  Not a MEX runtime; nothing here is linked or run. */
#ifndef KWB_TEST_MEX_STUB_H
#define KWB_TEST_MEX_STUB_H
#include <stddef.h>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum {
  mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
  mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
  mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS, mxFUNCTION_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;

mxArray* mxGetField(const mxArray* pm, mwIndex index, const char* fieldname);
void mxSetField(mxArray* pm, mwIndex index, const char* fieldname, mxArray* value);
void* mxGetData(const mxArray* pm);
size_t mxGetNumberOfElements(const mxArray* pm);
double mxGetScalar(const mxArray* pm);
mxClassID mxGetClassID(const mxArray* pm);
int mxIsEmpty(const mxArray* pm);
int mxIsNumeric(const mxArray* pm);
int mxIsLogical(const mxArray* pm);
int mxIsSingle(const mxArray* pm);
int mxIsDouble(const mxArray* pm);
int mxIsStruct(const mxArray* pm);
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID classid, mxComplexity flag);
mxArray* mxCreateNumericMatrix(mwSize m, mwSize n, mxClassID classid, mxComplexity flag);
mxArray* mxCreateStructMatrix(mwSize m, mwSize n, int nfields, const char** fieldnames);
void* mxMalloc(size_t n);
void mxFree(void* ptr);
void mexErrMsgIdAndTxt(const char* errorid, const char* errormsg, ...);

#endif
