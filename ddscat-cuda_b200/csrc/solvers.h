// Solver interface shared by the C ABI and the solver implementations.
#pragma once
#include "engine.h"

namespace ddb {

template <typename T> struct SolveIO {
  Engine<T>* eng = nullptr;
  VecOps<T>* ops = nullptr;
  cudaStream_t stream = 0;
  int n = 0;                        // 3*NAT0
  const cplx<T>* b = nullptr;       // compact right-hand side
  cplx<T>* x = nullptr;             // compact: initial guess in, solution out
  const cplx<T>* adia = nullptr;    // CXADIA (layout a_full)
  const cplx<T>* aoff = nullptr;    // CXAOFF or null
  int a_full = 1;
  const cplx<T>* adia_full = nullptr;  // CXADIA in the full layout (PBCGST's DIAGL preconditioner)
  cplx<T>* work = nullptr;          // 13*n scratch
  cplx<T>* sy = nullptr;            // n: MATVEC output staging
  int maxit = 0;
  double tol = 0.0;
  int verbose = 0;
  int itno = 0;
  double tole = 0.0;
  int ncompte = 0;
};

// one reference-style console line for a MATVEC of GPU time gpu_ms (cu:417)
void report_matvec_line(int cwhat, const char* path, float gpu_ms);

template <typename T> int solve_pbcgs2(SolveIO<T>& io);
template <typename T> int solve_qmrccg(SolveIO<T>& io);
template <typename T> int solve_pbcgst(SolveIO<T>& io);
template <typename T> int solve_petrkp(SolveIO<T>& io);
template <typename T> int solve_gpbicg(SolveIO<T>& io);
template <typename T> int solve_bicgstab4(SolveIO<T>& io);
template <typename T> int solve_gpbicgstab2(SolveIO<T>& io);
template <typename T> int solve_gpbicgstab4(SolveIO<T>& io);

// post-processing (post.cu)
template <typename T>
int evalq_compute(Engine<T>& eng, VecOps<T>& ops, const cplx<T>* e, const cplx<T>* p, const cplx<T>* adia,
                  const cplx<T>* aoff, int a_full, cplx<T>* qbuf, double ak3, double2* zabs, double2* zep);

struct FarDir {
  double k[3];
};
// S[d][c] = sum_j P_c(j) exp(-i k_d . r_j), r_j = ((i+1)+x0)*dx; FP64 sums.
template <typename T>
int farfield_sums(Engine<T>& eng, const cplx<T>* p, const float* dirs_host, int ndir, const float dx[3], const float x0[3],
                  double2* sums_host, cudaStream_t s);

// S and the position moments of the scattered angular-momentum flux:
// sums[d][0..2] = S_a, sums[d][3 + 3a + b] = U_ab = sum_j P_a(j) r_jb exp(-i k_d . r_j)
// (k_d given in FP64); FP32 phases and per-thread sums, FP64 block sums.
template <typename T>
int farfield_torque_sums(Engine<T>& eng, const cplx<T>* p, const double* dirs_host, int ndir, const float dx[3],
                         const float x0[3], double2* sums_host, cudaStream_t s);
// Torque of the incident field e on the dipoles p (both compact, device):
// gamma[0..2] = sum 1/2 Re(P x conj(E)), gamma[3..5] = sum (1/2) Im(P.conj(E)) r x k.
template <typename T>
int incident_torque(Engine<T>& eng, const cplx<T>* p, const cplx<T>* e, const float dx[3], const float x0[3],
                    const double k[3], double gamma[6], cudaStream_t s);

// The same sums with FP64 phases and FP64 accumulation (all-FP64 amplitudes);
// occ: compact -> site map of the grid, p: compact complex-double polarisation.
int farfield_sums_f64(const int* occ, int nx, int ny, int nz, int nat0, const double2* p, const double* dirs_host,
                      int ndir, const double dx[3], const double x0[3], double2* sums_host, cudaStream_t s);

// Amplitude and Mueller matrices per scattering direction from f_ml (host in / out).
int mueller_compute(int ndir, const float* ak, const float2* e01, const float2* e02, const float* em2,
                    const float2* f11, const float2* f21, const float2* f12, const float2* f22, float2* s_out,
                    double* m_out);
int mueller_compute_f64(int ndir, const double* ak, const double2* e01, const double2* e02, const double* em2,
                        const double2* f11, const double2* f21, const double2* f12, const double2* f22,
                        double2* s_out, double* m_out);

}  // namespace ddb
