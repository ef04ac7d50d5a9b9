/*
 * cufft.h (host stand-in) -- the four cuFFT calls the reference makes
 * (src/cu/pressure.cu:527-548), implemented on the CPU with oracle/cpu_fft.c.
 * TEST INFRASTRUCTURE ONLY: it shadows the toolkit header only for the host
 * build of the reference's sources under oracle/_ref.
 */
#ifndef WF_SHIM_CUFFT_H
#define WF_SHIM_CUFFT_H

#include <cuComplex.h>

typedef int cufftHandle;
typedef enum { CUFFT_SUCCESS = 0, CUFFT_INVALID_PLAN = 1, CUFFT_ALLOC_FAILED = 2, CUFFT_INVALID_VALUE = 4 } cufftResult;
typedef enum { CUFFT_Z2Z = 0x69 } cufftType;
#define CUFFT_FORWARD -1
#define CUFFT_INVERSE 1
typedef cuDoubleComplex cufftDoubleComplex;

cufftResult cufftPlanMany(cufftHandle *plan, int rank, int *n, int *inembed, int istride, int idist,
                          int *onembed, int ostride, int odist, cufftType type, int batch);
cufftResult cufftPlan2d(cufftHandle *plan, int nx, int ny, cufftType type);
cufftResult cufftExecZ2Z(cufftHandle plan, cufftDoubleComplex *idata, cufftDoubleComplex *odata, int direction);
cufftResult cufftDestroy(cufftHandle plan);

#endif
