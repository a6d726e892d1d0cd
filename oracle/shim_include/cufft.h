/* CPU stand-in for the two cuFFT entry points the reference calls
 * (cufftPlan2d, cufftExecC2C; functions/useful_functions.cpp:646-660 and
 * main_code/run_with_active_gels.cpp:87-88).  Test infrastructure only: it lets
 * the reference's own C++ sources run serially on the host as the oracle.
 * PFAG_REF_DOUBLE selects the FP64 build, where the complex type holds doubles
 * (the float->double rewritten reference copy). */
#ifndef PFAG_SHIM_CUFFT_H
#define PFAG_SHIM_CUFFT_H
#ifdef __cplusplus
extern "C" {
#endif
typedef int cufftHandle;
typedef enum { CUFFT_SUCCESS = 0, CUFFT_INVALID_PLAN = 1, CUFFT_ALLOC_FAILED = 2,
               CUFFT_INVALID_VALUE = 4, CUFFT_EXEC_FAILED = 6 } cufftResult;
typedef enum { CUFFT_C2C = 0x29 } cufftType;
#define CUFFT_FORWARD -1
#define CUFFT_INVERSE 1
#ifdef PFAG_REF_DOUBLE
typedef struct { double x, y; } cufftComplex;
#else
typedef struct { float x, y; } cufftComplex;
#endif
cufftResult cufftPlan2d(cufftHandle *plan, int nx, int ny, cufftType type);
cufftResult cufftExecC2C(cufftHandle plan, cufftComplex *idata, cufftComplex *odata, int direction);
cufftResult cufftDestroy(cufftHandle plan);
#ifdef __cplusplus
}
#endif
#endif
