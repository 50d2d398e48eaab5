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

/* Number of CUDA kernels this library has launched since it was loaded. */
DDSCAT_CUDA_API unsigned long long ddscat_b200_launch_count(void);

/* Times the device-resident MATVEC of the prepared target: nrhs right-hand
 * sides per call (compact layout, per-RHS CXADIA, no CXAOFF), `iters` calls
 * after 3 warm-up calls, CUDA events on the library stream.  Writes the mean
 * milliseconds per call.  Allocates its own scratch vectors.  Codes: 400
 * invalid / not prepared, 401 allocation, 402 CUDA failure. */
DDSCAT_CUDA_API int ddscat_b200_matvec_timing(int nrhs, int iters, int cwhat, float *ms_per_call);

/* FFT launch-shape autotuner for the prepared target: times `iters` MATVECs
 * (after two warm-up calls) under every launch shape that changes a kernel the
 * grid uses (register-pass block sizes and y-pass columns per block on
 * power-of-two axes, generic Stockham tile sizes on the others; the x-first
 * pipeline of all-power-of-two grids has none) and keeps the fastest for the
 * rest of the target's life.  Writes the default and the chosen shape's time
 * per call.  Codes: 410 invalid argument / not prepared, 411 failure. */
DDSCAT_CUDA_API int ddscat_b200_autotune_f32(int iters, float *default_ms, float *best_ms);

/* Batched solve of nrhs systems A_r x_r = b_r that share the prepared target
 * and Green tensor (same |k|; CXADIA/CXAOFF may differ per right-hand side,
 * e.g. per orientation and polarisation).  b, x (initial guess in, solution
 * out), adia and aoff are arrays of nrhs full vectors (3*NAT complex float
 * each, RHS r at element offset r*3*NAT), all host pointers or all device
 * pointers; aoff may be NULL (no off-diagonal site blocks).  Each RHS follows
 * the recurrence of the single-RHS entry point of the same solver (reliable
 * residual every 20 iterations, restart policy, MATVEC count); every kernel
 * launch covers all RHS still iterating.  Per-RHS outputs: itno, tole
 * (achieved true relative residual), ncompte, status (0, or the error code
 * the single-RHS entry point would have returned for that RHS).
 * solver: DDSCAT_B200_QMRCCG or DDSCAT_B200_PBCGS2, optionally OR'ed with
 * DDSCAT_B200_REPLACE_RESIDUAL: at a reliable-residual check that finds the
 * RHS unconverged with a large gap, replace the recursive residual by the
 * true one and keep the Krylov state, instead of restarting the solver from
 * the true residual (convergence is still declared on the true residual).
 * QMRCCG may also be OR'ed with DDSCAT_B200_QMR_SYMMETRIC: the reference's
 * QMRCCG starts its left and right Lanczos vectors equal (both r0) and the DDA
 * matrix is complex symmetric, so the left vectors stay equal to the right
 * ones and A p equals the recurrence vector q; this variant drops the second
 * MATVEC of each iteration (one MATVEC per iteration instead of two; same
 * iterates in exact arithmetic).  QMRCCG with both flags may add
 * DDSCAT_B200_GRAPH: the iterations then run device-driven (scalar
 * recurrences, masks and reliable-residual decisions in FP64 on the GPU) as a
 * captured CUDA graph with the reliable-residual check in a conditional node,
 * so an iteration makes no host round trip; the host reads the active-RHS
 * count every four graph launches.
 * Codes: 500 invalid argument / not prepared, 501 solver, 502 mixed pointer
 * kinds, 503 workspace allocation, 504 input transfer, 505 solver failure,
 * 506 output transfer. */
#define DDSCAT_B200_QMRCCG 1
#define DDSCAT_B200_PBCGS2 2
#define DDSCAT_B200_REPLACE_RESIDUAL 0x100
#define DDSCAT_B200_QMR_SYMMETRIC 0x200
#define DDSCAT_B200_INPUTS_F64 0x400
#define DDSCAT_B200_AUTOTUNE 0x800
#define DDSCAT_B200_GRAPH 0x1000

/* Polarisability prescriptions of ddscat_b200_make_inputs_pol_f32 (DDSCAT's
 * CMDPOL values). */
#define DDSCAT_B200_LATTDR 0
#define DDSCAT_B200_GKDLDR 1
#define DDSCAT_B200_FLTRCD 2
DDSCAT_CUDA_API int ddscat_b200_solve_batch_f32(int solver, int nrhs, const void *b, void *x, const void *adia,
                                                const void *aoff, int maxit, float tol, int *itno, float *tole,
                                                int *ncompte, int *status);

/* CUDA-event time spent in MATVECs during the last batched solve, the number
 * of single-RHS MATVECs it performed and the number of batched MATVEC calls. */
DDSCAT_CUDA_API int ddscat_b200_last_solve_stats(double *matvec_ms, long long *rhs_matvecs, int *matvec_calls);

/* FP64 true relative residuals ||b_r - A x_r|| / ||b_r|| with the operator
 * evaluated entirely in FP64 on the GPU (FP64 Green tensor, FP64 FFTs).
 * Arrays as in ddscat_b200_solve_batch_f32; aoff may be NULL.  Codes: 510
 * invalid, 511 FP64 engine setup, 512 transfer, 513 reduction. */
DDSCAT_CUDA_API int ddscat_b200_residual_f64(int nrhs, const void *b, const void *x, const void *adia,
                                             const void *aoff, double *resid);

/* MATVEC that allocates no device memory; no counterpart in the reference.
 * For callers that cannot call cudaMalloc where they need the operator
 * (real-time loops that forbid allocation once started, or applications that
 * hand all device memory to their own pool): y = A x (cwhat 'N') or A^H x
 * ('C') for the prepared target, with x, y, adia and aoff caller-owned DEVICE
 * vectors in the full layout of ddscat_cuda_apply_f32 (3*NAT complex floats;
 * aoff may be NULL), launched on `stream` (a cudaStream_t, NULL for the legacy
 * default stream), with the device of the prepare current.  The MATVEC
 * scratch is a fixed 48 MiB array (6,291,456 complex floats) in the library's
 * device image; every GPU that loads the library holds it until exit.  It must
 * hold 3*nz*Mx*ny + 3*My*nz*Mx complex floats for the padded FFT lengths Mx,
 * My of the prepared grid (18*NAT when M = 2n: unpadded targets up to
 * NAT = 349,525 sites, e.g. 64^3; padded grids need more), else the call
 * returns 601.  All calls share the array and it keeps the last call's
 * contents (nothing needs to start at zero); calls that overlap on the GPU
 * race, so serialise them.  The first call on a device (and the first after
 * each prepare) does one-time set-up and should come before any stream
 * capture.  Codes: 600 invalid argument, not prepared or another device
 * current, 601 target larger than the fixed scratch, 602 scratch address lookup
 * failed, 21-25 kernel launch failure. */
DDSCAT_CUDA_API int ddscat_b200_apply_noalloc_f32(int cwhat, const void *x, void *y, const void *adia,
                                                  const void *aoff, void *stream);

/* Amplitude matrix (S1..S4) and 4x4 Mueller matrix S_ij per scattering
 * direction, the step DDSCAT's GETMUELLER performs after SCAT (GETMUELLER is not
 * part of the reference; this restates the definitions of Bohren & Huffman 1983,
 * section 3.2 and eq. 3.16).  f11, f21 are the f1, f2 outputs of
 * ddscat_cuda_scat_f32 for incident polarisation e01; f12, f22 those for e02
 * (ndir complex floats each, same EM1/EM2 and AKS).  em2 (ndir x 3) is EM2 of
 * the SCAT call, in DDSCAT's convention EM2 = n x EM1 (phi-hat when EM1 is
 * theta-hat); Bohren & Huffman's perpendicular vector is -EM2, for incident and
 * scattered light, and e_par,i = khat x e_perp,i.
 * Outputs: s1234 (ndir x 4 complex floats S1, S2, S3, S4, may be NULL) and smat
 * (ndir x 16 doubles, S_ij row-major).  Host pointers.  Codes: 700 invalid
 * argument, 701 allocation, 702 transfer, 703 kernel launch. */
DDSCAT_CUDA_API int ddscat_b200_mueller_f32(int ndir, const float *ak, const void *e01, const void *e02,
                                            const float *em2, const void *f11, const void *f21, const void *f12,
                                            const void *f22, void *s1234, double *smat);

/* The same with complex-double amplitudes and FP64 vectors (s1234 ndir x 4
 * complex doubles): the Mueller matrix of an all-FP64 reference solve.  No
 * counterpart in the reference.  Codes as ddscat_b200_mueller_f32. */
DDSCAT_CUDA_API int ddscat_b200_mueller_f64(int ndir, const double *ak, const void *e01, const void *e02,
                                            const double *em2, const void *f11, const void *f21, const void *f12,
                                            const void *f22, void *s1234, double *smat);

/* All-FP64 scattering amplitudes f1, f2 of nrhs polarisations at ndir
 * directions, with the normalisation of the f1/f2 outputs of
 * ddscat_cuda_scat_f32 (|k|^3/sqrt(E02) sum_j EM . P_j exp(-i AKS . r_j),
 * r_j = ((i+1)+X0)*DX), but FP64 phases and FP64 sums: the reference values the
 * S_ij of an FP32 solve are checked against.  No counterpart in the reference
 * (its SCAT sums FP32 phases).  x: nrhs full component-major complex-double
 * polarisations (3*NAT each, host or device) of the prepared target; aks, em1,
 * em2: ndir x 3; f1, f2: nrhs x ndir complex doubles (host).  Codes: 710
 * invalid argument or not prepared, 711 allocation, 712 far-field sums. */
DDSCAT_CUDA_API int ddscat_b200_scat_amplitudes_f64(int nrhs, const void *x, int ndir, const double *ak,
                                                    const double *aks, const double *em1, const double *em2,
                                                    const double *dx, const double *x0, double e02, void *f1,
                                                    void *f2);

/* All-FP64 cross sections of SCAT's angular integration for nrhs
 * polarisations: Csca, Csca*g (3 per RHS), Csca*<cos^2 theta> and the
 * backscatter term, with the direction set and quadrature weights that
 * ddscat_cuda_scat_f32 builds from AK, CXE01 and ETASCA
 * (ddscat_matvec_cuda.cu:849-875, :957-1002), but FP64 phases and FP64 sums of
 * complex-double polarisations: the reference values that the Qsca and g of
 * an FP32 solve are checked against.  No counterpart in the reference.
 * x: nrhs full component-major complex-double polarisations (3*NAT each, host
 * or device) of the prepared target; e01: nrhs x 3 complex floats (CXE01_TF of
 * each RHS); outputs per RHS (host): cbksca[nrhs], csca[nrhs], cscag[3*nrhs],
 * cscag2[nrhs], navg[nrhs].  Codes: 710 invalid argument or not prepared, 711
 * allocation or transfer, 712 far-field sums. */
DDSCAT_CUDA_API int ddscat_b200_scat_csca_f64(int nrhs, const void *x, const float *ak, const void *e01,
                                              float etasca, const float *dx, const float *x0, float e02,
                                              double *cbksca, double *csca, double *cscag, double *cscag2,
                                              int *navg);

/* Radiative torque of the resident solution, DDSCAT's CMDTRQ = 'DOTORQ'
 * branch of SCAT (getfml_cuda.f90:1135-1144 sends it to DDSCAT's CPU SCAT,
 * whose torque sums are not part of the reference).  Requires a resident
 * solution P and incident field E (after a solver call or a non-resident
 * EVALQ).  Outputs torque cross sections C = 8 pi k Gamma / E02 in the frame of
 * AK (divide by pi a_eff^2 for DDSCAT's Q_Gamma):
 *   ctrq_inc[3]  torque of the incident field on the induced dipoles,
 *                sum_j 1/2 Re(P_j x E_j*) + (1/2) Im(P_j . E_j*) r_j x k
 *                (the angular momentum removed from the incident beam);
 *   ctrq_flux[3] angular momentum carried off by the scattered light, the
 *                far-field flux integrated over SCAT's ETASCA direction set;
 *   net radiative torque = ctrq_inc - ctrq_flux.
 * r_j = ((i+1)+X0)*DX as in SCAT; the direction set and navg as in
 * ddscat_cuda_scat_f32 for AK, CXE01 and ETASCA.  Codes: 340 invalid
 * state/argument, 341-343 incident-torque workspace/kernel/transfer, 344 bad
 * CXE01, 345/322/329 far-field sums. */
DDSCAT_CUDA_API int ddscat_b200_scat_torque_f32(const float *ak, const float *dx, float e02, float etasca,
                                                const void *e01, const float *x0, double *ctrq_inc,
                                                double *ctrq_flux, int *navg);

/* Right-hand sides and CXADIA for nrhs incident waves, generated on the GPU
 * for the prepared target (DDSCAT computes them on the host in EVALE and
 * ALPHADIAG; no counterpart in the reference ABI).  k: nrhs x 3 wave vectors in
 * lattice units; e0: nrhs x 3 complex polarisations; x0: the SCAT origin
 * offset (r_j = (ix+1, iy+1, iz+1) + x0); m: nmat complex refractive indices;
 * icomp: NAT material indices 1..nmat (0 = vacuum) or NULL for material 1 on
 * every occupied site.  Writes b = e0 exp(i k.r_j) on occupied sites (0 on
 * vacuum) and adia = 1/alpha_LDR (Draine & Goodman 1993) of each site's
 * material, as nrhs full vectors (3*NAT complex floats each, the input layout
 * of ddscat_b200_solve_batch_f32); either output may be NULL; both host or both
 * device pointers.  Codes: 610 invalid argument / not prepared, 611 material
 * index out of range, 612 allocation or transfer, 613 kernel failure. */
DDSCAT_CUDA_API int ddscat_b200_make_inputs_f32(int nrhs, const float *k, const void *e0, const float *x0, int nmat,
                                                const void *m, const int16_t *icomp, void *b, void *adia);

/* ddscat_b200_make_inputs_f32 with a choice of polarisability prescription
 * (DDSCAT's CMDPOL; ALPHADIAG is not part of the reference, so the formulas
 * are restated from the publications; lattice units d = 1, 1/alpha_CM =
 * (4 pi/3)(m^2+2)/(m^2-1), b1 = -1.891531, b2 = 0.1648469, b3 = -1.7700004):
 *   DDSCAT_B200_LATTDR  1/alpha = 1/alpha_CM + (b1 + m^2 b2 + m^2 b3 S)(kd)^2
 *                       - (2/3) i (kd)^3, S = sum_a (khat_a Re e_a)^2 (Draine &
 *                       Goodman 1993), the same for the three components;
 *   DDSCAT_B200_GKDLDR  component c with S replaced by khat_c^2
 *                       (Gutkowicz-Krusin & Draine 2004): CXADIA differs per
 *                       component and does not depend on the polarisation;
 *   DDSCAT_B200_FLTRCD  1/alpha = 1/alpha_CM - (4/3)(kd)^2 - (2/(3 pi))
 *                       ln((pi - kd)/(pi + kd)) (kd)^3 - (2/3) i (kd)^3, kd < pi
 *                       (filtered coupled dipoles, Piller & Martin 1998,
 *                       Gay-Balmaz & Martin 2002).
 * Other arguments and codes as ddscat_b200_make_inputs_f32 (610 also for an
 * unknown cmdpol or FLTRCD with kd >= pi). */
DDSCAT_CUDA_API int ddscat_b200_make_inputs_pol_f32(int cmdpol, int nrhs, const float *k, const void *e0,
                                                    const float *x0, int nmat, const void *m, const int16_t *icomp,
                                                    void *b, void *adia);

/* All-FP64 batched solve: the recurrence of ddscat_b200_solve_batch_f32 (same
 * solver codes and flags) with complex-double vectors, an FP64 Green tensor and
 * FP64 FFTs, as the reference solution against which FP32 results (Q values,
 * residuals) are checked.  b, adia, aoff: nrhs complex-float full vectors (as
 * for the FP32 entry point, widened on the GPU); x: nrhs complex-DOUBLE full
 * vectors, initial guess in, solution out; all host or all device pointers.
 * With DDSCAT_B200_INPUTS_F64 OR'ed into solver, b, adia and aoff are
 * complex-double full vectors too.
 * tole is the achieved true relative residual.  Codes: 520 invalid argument /
 * not prepared, 521 solver or flag, 522 mixed pointer kinds, 523 workspace,
 * 524 input transfer, 525 solver failure, 526 output transfer; a breakdown of
 * any RHS returns that RHS's status code. */
DDSCAT_CUDA_API int ddscat_b200_solve_batch_f64(int solver, int nrhs, const void *b, void *x, const void *adia,
                                                const void *aoff, int maxit, double tol, int *itno, double *tole,
                                                int *ncompte, int *status);

/* Adjoint gradient (no counterpart in the reference).  For nrhs forward
 * solutions P_r of A_r P_r = E_r and adjoint sources s_r, solves the adjoint
 * systems A_r lam_r = s_r (A^T = A: the same complex-symmetric operator, one
 * batched one-MATVEC QMRCCG solve with residual replacement, tolerance tol) and
 * returns per site j the derivative of the holomorphic functional F_r = s_r^T P_r
 * with respect to a site parameter that enters A only through CXADIA:
 *   grad[r][j] = -sum_c lam_r[c][j] * dadia_r[c][j] * P_r[c][j],
 * dadia_r = dCXADIA/dparameter (e.g. the derivative of the LDR 1/alpha with
 * respect to the permittivity).  s_r = conj(E_r) gives dCext: Cext = 4 pi k
 * Im(F)/E02; s_r = the far-field weights of ddscat_cuda_scat_f32 gives the
 * derivative of a scattering amplitude.  p, src, adia, dadia, lam (optional):
 * nrhs full vectors (3*NAT complex floats); grad: nrhs x NAT complex floats
 * (zero on vacuum sites); all host or all device pointers.  itno / tole: the
 * adjoint solves' iterations and achieved residuals.  Codes: 530 invalid
 * argument / not prepared, 531 mixed pointer kinds, 532 workspace, 533 input
 * transfer, 534 solver failure, 535 gradient or output failure. */
DDSCAT_CUDA_API int ddscat_b200_adjoint_f32(int nrhs, const void *p, const void *src, const void *adia,
                                            const void *dadia, int maxit, float tol, void *grad, void *lam, int *itno,
                                            float *tole);

/* Adjoint gradient with the forward field recomputed, not stored (no
 * counterpart in the reference).  For one incident field E (full vector) and
 * nsrc adjoint sources s_k, solves the forward system A P = E and the adjoint
 * systems A lam_k = s_k together (they share the operator; one batched
 * one-MATVEC QMRCCG solve with residual replacement, nsrc + 1 right-hand
 * sides) and returns grad[k][j] = -sum_c lam_k[c][j] dadia[c][j] P[c][j], the
 * derivative of F_k = s_k^T P with respect to a site parameter entering only
 * CXADIA.  The caller never holds P: for large grids it costs one extra
 * right-hand side inside the call instead of a stored full vector.  e, adia,
 * dadia: one full vector each (3*NAT complex floats); src: nsrc full vectors;
 * grad: nsrc x NAT complex floats (zero on vacuum sites); p: optional output of
 * the forward solution (full vector) or NULL; itno / tole: nsrc + 1 entries,
 * the forward solve first.  All host or all device pointers.  Codes as
 * ddscat_b200_adjoint_f32. */
DDSCAT_CUDA_API int ddscat_b200_adjoint_fwd_f32(int nsrc, const void *e, const void *src, const void *adia,
                                                const void *dadia, int maxit, float tol, void *grad, void *p,
                                                int *itno, float *tole);

/* Far-field adjoint sources built on the GPU (no counterpart in the
 * reference): for nw scattering wave vectors aks (nw x 3, |aks| = |k|) and
 * basis vectors em (nw x 3), the full vectors
 *   w_k[c][j] = |aks_k|^3 / sqrt(e02) em_k[c] exp(-i aks_k . r_j)
 * on occupied sites (0 on vacuum), r_j = (ix+1, iy+1, iz+1) + x0 (unit
 * spacing), so that w_k^T P is the scattering amplitude f of
 * ddscat_cuda_scat_f32 along em_k (cu:957-1002).  FP64 phases, complex-float
 * output: w is nw x 3*NAT complex floats, host or device.  Codes: 720 invalid
 * argument or not prepared, 721 allocation or transfer, 722 kernel failure. */
DDSCAT_CUDA_API int ddscat_b200_ffweights_f32(int nw, const double *aks, const double *em, const double *x0,
                                              double e02, void *w);

/* Many targets of uneven size solved together (no counterpart in the
 * reference, whose state holds one target).  Target t has lattice dims[3t..3t+2],
 * occupancy iocc[t] (int16, NAT_t), wave vector ak[3t..3t+2] (lattice units;
 * point dipoles, IPBC = 0, unit spacing) and nrhs[t] right-hand sides: b[t],
 * x[t] (initial guess in, solution out) and adia[t] are host arrays of nrhs[t]
 * full vectors (3*NAT_t complex floats each).  Each target gets its own
 * engine, Green tensor and CUDA stream; nthreads host threads (0: up to 8)
 * drive the targets' batched solves concurrently, largest first.  solver and
 * flags as for ddscat_b200_solve_batch_f32, plus DDSCAT_B200_AUTOTUNE: tune each
 * target's FFT launch shapes before its solve (see ddscat_b200_autotune_f32);
 * per-RHS outputs in target order.
 * The FFT3D layout is used in both libraries.  Codes: 540 invalid argument,
 * 541 solver or flag, 542 workspace, 543 geometry or Green build, 544 input
 * transfer, 545 solver failure, 546 output transfer; a breakdown returns that
 * RHS's status code. */
DDSCAT_CUDA_API int ddscat_b200_multi_solve_f32(int ntarget, const int *dims, const int16_t *const *iocc,
                                                const float *ak, const int *nrhs, const void *const *b, void *const *x,
                                                const void *const *adia, int solver, int maxit, float tol,
                                                int nthreads, int *itno, float *tole, int *ncompte, int *status);

#ifdef __cplusplus
}
#endif
