// Batched multi-RHS Krylov solves (library extension, no reference counterpart).
//
// R independent systems A_r x_r = b_r share one prepared Green tensor (same
// target and |k|; CXADIA/CXAOFF may differ per RHS, e.g. per polarisation).
// Vectors are compact (3*NAT0) and stored RHS-major: RHS r of vector v at
// v + r*n.  Every vector kernel and every MATVEC pass covers all RHS in one
// launch; a per-RHS mask skips RHS that converged, broke down or are not in
// the current sub-step, so each RHS follows exactly the single-RHS recurrence.
#pragma once
#include <vector>
#include "engine.h"

namespace ddb {

template <typename T> struct BatchOps {
  using C = cplx<T>;
  cudaStream_t stream = 0;
  int R = 0;           // number of RHS
  int n = 0;           // 3*NAT0
  int nb = 0;          // reduction blocks per RHS
  double2* d_part = nullptr;   // [R][K][nb]
  double2* d_out = nullptr;    // [R][K]
  unsigned* d_cnt = nullptr;   // [R]
  double2* h_out = nullptr;    // pinned [R][K]
  double2* h_coef = nullptr;   // pinned ring of coefficients
  double2* d_coef = nullptr;
  size_t coef_cap = 0, coef_pos = 0;
  int* h_mask = nullptr;       // pinned staging for masks
  int* d_masks = nullptr;      // device mask slots [MASKS][R]
  size_t mask_pos = 0;
  static constexpr int KMAX = 8;
  static constexpr int MASKS = 64;

  int init(int R_, int n_, cudaStream_t s);
  void release();
  // upload a per-RHS mask (nonzero = active); returns the device pointer
  const int* mask(const std::vector<int>& m);
  // d_r = zd_r d_r + za_r a_r + zb_r b_r over RHS with mask_r != 0;
  // coefficient arrays have R entries (null array = term absent)
  int lin(C* d, const double2* zd, const C* a, const double2* za, const C* b, const double2* zb, const int* mask);
  int copy(C* d, const C* a, const int* mask);
  int zero(C* d, const int* mask);
  // K inner products per RHS: conj[k] ? sum conj(a_k) b_k : sum a_k b_k ; results [R][K] on the host
  int dots(int K, const C* const* a, const C* const* b, const int* conj, const int* mask, std::vector<double2>& out);
  // ||a - b||^2 and ||a - b - c||^2 per RHS (FP64)
  int diff_norms(const C* a, const C* b, const C* c, const int* mask, std::vector<double2>& out);
  // fused steps of the one-MATVEC QMRCCG iteration (see kq_pqv / kq_dsxr):
  // qmr_pqv leaves |vt|^2 and vt^T vt in output slots 2 and 3 (read them with
  // slot() after the next synchronising call); qmr_dsxr returns |r|^2 per RHS
  int qmr_pqv(C* p, C* q, C* vt, const C* atw, const double2* cp, const double2* cv, const double2* cq,
              const double2* cw, const double2* ct, const int* mask);
  int qmr_dsxr(C* d, C* s, C* x, C* r, const C* p, const C* q, const double2* th, const double2* ka,
               const int* mask, std::vector<double2>& rr);
  double2 slot(int r, int k) const { return h_out[(size_t)r * 8 + k]; }
  const double2* upload(const std::vector<const double2*>& cols);
  // after a stream sync every pending coefficient copy has landed; masks wrap on
  // their own (a mask pointer stays valid for MASKS-1 further uploads)
  void reset_ring() { coef_pos = 0; }
};

struct BatchResult {
  std::vector<int> itno, ncompte, status;
  std::vector<double> tole;
};

template <typename T> struct BatchIO {
  Engine<T>* eng = nullptr;
  BatchOps<T>* ops = nullptr;
  int R = 0, n = 0;
  const cplx<T>* b = nullptr;     // [R][n]
  cplx<T>* x = nullptr;           // [R][n] initial guess in, solution out
  const cplx<T>* adia = nullptr;  // [R][n] compact
  const cplx<T>* aoff = nullptr;  // [R][n] compact or null
  cplx<T>* work = nullptr;        // [nwork][R][n]
  int nwork = 0;
  int maxit = 0;
  double tol = 0.0;
  int verbose = 0;
  // Reliable-residual policy at a check that finds no convergence: 0 restarts
  // the Krylov process from the true residual when the gap test fails (the
  // single-RHS entry points); 1 replaces the recursive residual by the true
  // one and keeps the Krylov state (residual replacement).
  int replace = 0;
  // QMRCCG only: 1 = one MATVEC per iteration (left Lanczos vectors equal the
  // right ones since A^T = A and both start from r0), 0 = the reference's
  // two-product form.
  int sym = 0;
  // QMRCCG with sym and replace: 1 = device-driven iterations launched as a
  // CUDA graph (no host round trip per iteration)
  int graph = 0;
  // PBCGS2 with graph (FP32): a multi-target group (pg_group_create) whose
  // coordinator runs the device-driven iterations of every member target as
  // branches of one graph; group_joined is set once this solve handed over (or
  // left the group)
  void* group = nullptr;
  int group_joined = 0;
  double matvec_ms = 0.0;         // CUDA-event time of the MATVECs inside the solve
  long long matvec_rhs = 0;       // RHS-MATVECs performed
  int matvec_calls = 0;
};

template <typename T> int solve_batch_qmrccg(BatchIO<T>& io, BatchResult& res);
// Multi-target graph group of FP32 batched PBCGS2 solves (see BatchIO::group):
// every member solve runs on its own host thread and either hands its graph
// iteration over (and blocks until the combined run ends) or leaves; the
// coordinator's pg_group_run waits for all `expected` members, then launches
// one graph whose branches are the members' iterations, once per Krylov step.
void* pg_group_create(int expected);
int pg_group_run(void* group);
void pg_group_leave(void* group);
void pg_group_destroy(void* group);
template <typename T> int solve_batch_pbcgs2(BatchIO<T>& io, BatchResult& res);
constexpr int BATCH_WORK_VECTORS = 12;

}  // namespace ddb
