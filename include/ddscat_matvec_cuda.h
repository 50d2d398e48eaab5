/* Drop-in C ABI of the B200 DDA library.
 *
 * Each declaration has the exact signature of the entry point with the same
 * name in the reference header ddscat_cuda_unified/cuda/ddscat_matvec_cuda.h,
 * which the reference loader dlsym()s (ddscat_cuda_unified/cuda/
 * ddscat_cuda_loader.c:62-80) and the Fortran bridge calls
 * (ddscat_cuda_unified/fortran/cuda_matvec_bridge.f90:14-115).  Host vectors are
 * complex float, full-grid, component-major v[j + m*NAT],
 * j = ix + NX*(iy + NY*iz); CXAOFF holds (a23, a31, a12) per site.  Every call
 * returns 0 on success and a nonzero code (the reference's codes) on failure,
 * with a message available from ddscat_cuda_last_error().  The library is not
 * thread-safe and works on the current CUDA device, like the reference.
 */
#pragma once
#include <stdint.h>
#ifdef _WIN32
#define DDSCAT_CUDA_API __declspec(dllexport)
#else
#define DDSCAT_CUDA_API __attribute__((visibility("default")))
#endif
#ifdef __cplusplus
extern "C" {
#endif

/* Builds the FFT'd Green tensor on the GPU and allocates the runtime.
 * Replaces ddscat_matvec_cuda.h:11-13 / ddscat_matvec_cuda.cu:1005-1017.
 * Codes: 201 invalid argument, 202 GAMMA<=0 with IPBC=1, 204 allocation,
 * 208 IOCC count != NAT0, 220+k Green build failure k. */
DDSCAT_CUDA_API int ddscat_cuda_prepare_green_f32(int nx, int ny, int nz, int ipbc, int nat, int nat0, int idipint,
                                                  float gamma, float pyd, float pzd, float akx, float aky, float akz,
                                                  float dx1, float dx2, float dx3, const int16_t *iocc);

/* Uses a CPU-supplied Green tensor (CXZC layout: IPBC=0 octant
 * (NX+1)(NY+1)(NZ+1)x6, IPBC=1 full 8*NAT x6).
 * Replaces ddscat_matvec_cuda.h:14-15 / ddscat_matvec_cuda.cu:1018-1026.
 * Codes: 1 invalid, 2 allocation, 4 Green H2D, 6 IOCC count != NAT0. */
DDSCAT_CUDA_API int ddscat_cuda_prepare_f32(int nx, int ny, int nz, int ipbc, int nat, int nat0, const void *green,
                                            const int16_t *iocc);

/* y = A x (cwhat='N') or A^H x (cwhat='C'), full host vectors.
 * Replaces ddscat_matvec_cuda.h:16-17 / ddscat_matvec_cuda.cu:1027-1029.
 * Codes: 10 not prepared, 11 invalid, 12-14 H2D, 15 D2H, 21-25 MATVEC launch, 26 a tile copy of the
 * MATVEC's x or y passes did not complete within its bounded wait (also returned by the solvers, the batched
 * solve and the MATVEC timing entry point when it happens during their MATVECs). */
DDSCAT_CUDA_API int ddscat_cuda_apply_f32(int cwhat, const void *x, void *y, const void *adia, const void *aoff);

/* Krylov solvers: b, x (initial guess in, solution out), adia, aoff are full
 * host vectors of ndim = 3*NAT; *itno iterations, *tole achieved relative
 * residual, *ncompte MATVEC count.  Replace ddscat_matvec_cuda.h:18-41 /
 * ddscat_matvec_cuda.cu:1031-1570 with the same error codes:
 * GPBICG 29-40, QMRCCG 29/50-61, PBCGST 29/70-87 (87 = MAXIT reached, x still
 * returned), PBCGS2 29/90-107 (MAXIT is not an error), PETRKP 29/110-124,
 * BiCGStab(4) 130-145, GPBiCGStab(2) 150-173, GPBiCGStab(4) 180-207. */
DDSCAT_CUDA_API int ddscat_cuda_solve_gpbicg_f32(const void *b, void *x, const void *adia, const void *aoff, int ndim,
                                                 int maxit, float tol, int *itno, float *tole, int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_qmrccg_f32(const void *b, void *x, const void *adia, const void *aoff, int ndim,
                                                 int maxit, float tol, int *itno, float *tole, int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_pbcgst_f32(const void *b, void *x, const void *adia, const void *aoff, int ndim,
                                                 int maxit, float tol, int *itno, float *tole, int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_pbcgs2_f32(const void *b, void *x, const void *adia, const void *aoff, int ndim,
                                                 int maxit, float tol, int *itno, float *tole, int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_petrkp_f32(const void *b, void *x, const void *adia, const void *aoff, int ndim,
                                                 int maxit, float tol, int *itno, float *tole, int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_bicgstab4_f32(const void *b, void *x, const void *adia, const void *aoff,
                                                    int ndim, int maxit, float tol, int *itno, float *tole,
                                                    int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_gpbicgstab2_f32(const void *b, void *x, const void *adia, const void *aoff,
                                                      int ndim, int maxit, float tol, int *itno, float *tole,
                                                      int *ncompte);
DDSCAT_CUDA_API int ddscat_cuda_solve_gpbicgstab4_f32(const void *b, void *x, const void *adia, const void *aoff,
                                                      int ndim, int maxit, float tol, int *itno, float *tole,
                                                      int *ncompte);

/* Cabs, Cext, Cpha from the resident solution (use_resident=1) or from compact
 * host arrays of 3*NAT0.  Replaces ddscat_matvec_cuda.h:42-44 /
 * ddscat_matvec_cuda.cu:919-955.  Codes 300-307. */
DDSCAT_CUDA_API int ddscat_cuda_evalq_f32(int use_resident, const void *e_compact, const void *p_compact,
                                          const void *adia_compact, const void *aoff_compact, float akx, float aky,
                                          float akz, float e02, double *cabs, double *cext, double *cpha);

/* Far-field sums of the resident solution: Csca, Csca*g(3), Csca*<cos^2>,
 * backscatter and f1/f2 at ndir selected directions.  Replaces
 * ddscat_matvec_cuda.h:45-49 / ddscat_matvec_cuda.cu:957-1002.  Codes 320-333. */
DDSCAT_CUDA_API int ddscat_cuda_scat_f32(int jpbc, int ndir, const float *ak, const float *aks, const float *dx,
                                         const float *em1, const float *em2, float e02, float etasca, const void *e01,
                                         const float *x0, double *cbksca, double *csca, double *cscag, double *cscag2,
                                         int *navg, void *f1, void *f2);

/* Frees all device state.  Replaces ddscat_matvec_cuda.h:50 / ddscat_matvec_cuda.cu:915. */
DDSCAT_CUDA_API int ddscat_cuda_release(void);

/* Text of the last error.  Replaces ddscat_matvec_cuda.h:51 / ddscat_matvec_cuda.cu:916. */
DDSCAT_CUDA_API const char *ddscat_cuda_last_error(void);

#ifdef __cplusplus
}
#endif
