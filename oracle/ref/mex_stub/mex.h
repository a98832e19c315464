/* Minimal stand-in for MATLAB's mex.h (test infrastructure only).
 *
 * The reference's simulation header (src/tem_simulation.cuh:34) includes its MATLAB glue
 * (src/matlab_mex.cuh), which needs these MATLAB C API names to compile. The oracle driver never
 * calls them: it fills the reference's Input_Multislice directly, like the reference's GUI entry
 * (gui_multem/multem.cu:28-50). The definitions below exist only to satisfy the linker and abort
 * if ever reached. */
#ifndef MT_ORACLE_MEX_STUB_H
#define MT_ORACLE_MEX_STUB_H

#include <cstddef>
#include <cstdio>
#include <cstdlib>

typedef struct mxArray_tag mxArray;
typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

[[noreturn]] inline void mt_mex_stub_abort(const char* name) {
    std::fprintf(stderr, "mex stub: %s called outside MATLAB\n", name);
    std::abort();
}

inline mxArray* mxGetField(const mxArray*, mwIndex, const char*) { mt_mex_stub_abort("mxGetField"); }
inline void mxSetField(mxArray*, mwIndex, const char*, mxArray*) { mt_mex_stub_abort("mxSetField"); }
inline double mxGetScalar(const mxArray*) { mt_mex_stub_abort("mxGetScalar"); }
inline size_t mxGetM(const mxArray*) { mt_mex_stub_abort("mxGetM"); }
inline size_t mxGetN(const mxArray*) { mt_mex_stub_abort("mxGetN"); }
inline double* mxGetPr(const mxArray*) { mt_mex_stub_abort("mxGetPr"); }
inline double* mxGetPi(const mxArray*) { mt_mex_stub_abort("mxGetPi"); }
inline bool mxIsStruct(const mxArray*) { mt_mex_stub_abort("mxIsStruct"); }
inline mxArray* mxCreateDoubleMatrix(mwSize, mwSize, mxComplexity) { mt_mex_stub_abort("mxCreateDoubleMatrix"); }
inline mxArray* mxCreateStructArray(mwSize, const mwSize*, int, const char**) {
    mt_mex_stub_abort("mxCreateStructArray");
}
#define mexPrintf std::printf

#endif
