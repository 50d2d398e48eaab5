/* Extensions of the B200 DDA library beyond the reference ABI.
 *
 * These entry points have no counterpart in ddscat_cuda_unified/cuda/
 * ddscat_matvec_cuda.h; they are new symbols only, and the 15 reference entry
 * points in ddscat_matvec_cuda.h keep their behaviour.
 */
#pragma once
#include <stdint.h>
#include "ddscat_matvec_cuda.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Per-iteration progress lines on stdout (the reference always prints them;
 * here they are off unless level != 0 or DDSCAT_B200_VERBOSE is set). */
DDSCAT_CUDA_API int ddscat_b200_set_verbose(int level);

/* 0 for the FFT3D build (libddscat_matvec_cuda.so), 1 for the SLICES build
 * (libddscat_matvec_cuda_slice.so). */
DDSCAT_CUDA_API int ddscat_b200_layout(void);

/* Times the device-resident MATVEC of the prepared target: nrhs right-hand
 * sides per call (compact layout, per-RHS CXADIA, no CXAOFF), `iters` calls
 * after 3 warm-up calls, CUDA events on the library stream.  Writes the mean
 * milliseconds per call.  Allocates its own scratch vectors.  Codes: 400
 * invalid / not prepared, 401 allocation, 402 CUDA failure. */
DDSCAT_CUDA_API int ddscat_b200_matvec_timing(int nrhs, int iters, int cwhat, float *ms_per_call);

#ifdef __cplusplus
}
#endif
