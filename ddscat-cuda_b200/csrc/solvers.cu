// Krylov solvers behind the ddscat_cuda_solve_*_f32 entry points.
//
// Each routine restates the corresponding reference routine of
// ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu (line ranges at each
// function) on compact 3*NAT0 device vectors: FP32 vectors, FP64 recurrence
// scalars, FP64 inner products, the reliable-residual policy (true residual
// every 20 iterations and on claimed convergence, restart when the recursion
// gap >= 1e-3 or on false convergence, cu:543-556), the same MATVEC counting
// and the same error codes.  Scalars are combined on the host from the
// device-reduced inner products (one small D2H per product, no full-vector
// transfers inside the loops).
#include <chrono>
#include <complex>
#include "engine.h"
#include "solvers.h"

namespace ddb {

// Console line per MATVEC of the reference entry points (the reference's
// report_matvec, cu:417): a running count, CWHAT, the solver, the GPU time of
// the MATVEC (CUDA events, waited for) and the wall time since the previous
// MATVEC ended, minus the previous line's own printing time.
struct MatvecReport {
  unsigned long long count = 0;
  bool have_prev = false;
  std::chrono::steady_clock::time_point prev_end;
  double last_print_ms = 0.0;
  void line(char cw, const char* path, float gpu_ms) {
    ++count;
    const auto now = std::chrono::steady_clock::now();
    const auto p0 = now;
    if (have_prev) {
      double dt = std::chrono::duration<double, std::milli>(now - prev_end).count() - last_print_ms;
      if (dt < 0) dt = 0;
      std::printf("CUDA MATVEC %llu [%c,%s]: GPU=%.6f ms  prev_end->end=%.6f ms  outside=%.6f ms\n", count, cw, path,
                  (double)gpu_ms, dt, dt - gpu_ms);
    } else {
      std::printf("CUDA MATVEC %llu [%c,%s]: GPU=%.6f ms  prev_end->end=N/A\n", count, cw, path, (double)gpu_ms);
    }
    std::fflush(stdout);
    last_print_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - p0).count();
    prev_end = now;
    have_prev = true;
  }
};
static MatvecReport g_mv_report;
void report_matvec_line(int cwhat, const char* path, float gpu_ms) { g_mv_report.line((char)cwhat, path, gpu_ms); }

using Z = std::complex<double>;
static inline double2 dz(Z z) { return make_double2(z.real(), z.imag()); }
static inline Z zd(double2 v) { return Z(v.x, v.y); }

constexpr int RELIABLE_PERIOD = 20;
constexpr double RELIABLE_GAP = 1.0e-3;

template <typename T> struct Ctx {
  using C = cplx<T>;
  SolveIO<T>& io;
  int n;
  int nc = 0;
  int err = 0;
  const char* label = "device";
  cudaEvent_t ev[2] = {nullptr, nullptr};
  explicit Ctx(SolveIO<T>& s, const char* solver = "device") : io(s), n(s.n), label(solver) {
    if (io.verbose && (cudaEventCreate(&ev[0]) != cudaSuccess || cudaEventCreate(&ev[1]) != cudaSuccess)) {
      cudaGetLastError();
      ev[0] = ev[1] = nullptr;
    }
  }
  ~Ctx() {
    if (ev[0]) cudaEventDestroy(ev[0]);
    if (ev[1]) cudaEventDestroy(ev[1]);
  }
  cudaStream_t st() const { return io.stream; }
  int mv(const C* in, C* out, int conj = 0) {
    MvArgs<T> a;
    a.x = in; a.y = out; a.io_full = 0;
    a.adia = io.adia; a.aoff = io.aoff; a.a_full = io.a_full; a.conj = conj; a.nrhs = 1;
    const bool timed = io.verbose && ev[0];
    if (timed) cudaEventRecord(ev[0], st());
    int rc = io.eng->matvec(a);
    if (!rc) ++nc;
    if (!rc && timed) {
      float ms = 0.f;
      cudaEventRecord(ev[1], st());
      if (cudaEventSynchronize(ev[1]) == cudaSuccess && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess)
        g_mv_report.line(conj ? 'C' : 'N', label, ms);
      else
        cudaGetLastError();
    }
    return rc;
  }
  Z dotc(const C* a, const C* b) { return zd(io.ops->dotc(n, a, b, &err)); }
  Z dotu(const C* a, const C* b) { return zd(io.ops->dotu(n, a, b, &err)); }
  double nrm(const C* a) { return io.ops->nrm2(n, a, &err); }
  // d = zd*d + za*a + zb*b
  void lin(C* d, Z zdd, const C* a = nullptr, Z za = 0.0, const C* b = nullptr, Z zb = 0.0) {
    v_lincomb<T>(d, dz(zdd), a, dz(za), b, dz(zb), n, st());
  }
  void copy(C* d, const C* a) { v_copy<T>(d, a, n, st()); }
  void zero(C* d) { v_zero<T>(d, n, st()); }
  void diff(C* d, const C* a, const C* b) { v_diff<T>(d, a, b, n, st()); }
  C* w(int slot) { return io.work + (size_t)slot * n; }
  // cu:543-556
  int reliable(const char* name, const C* rhs, const C* xcur, const C* rrec, double rhsnorm, double recursive,
               double tol, double& true_res, bool& converged, bool& restart) {
    if (rhsnorm <= 0.0) { set_error(name, "reliable residual: zero RHS norm"); return 1; }
    int rc = mv(xcur, io.sy);
    if (rc) return rc;
    const double tr = io.ops->norm_diff(n, rhs, io.sy, &err);
    const double gapn = io.ops->norm_gap(n, rhs, io.sy, rrec, &err);
    if (err) return 1;
    true_res = tr / rhsnorm;
    const double gap = tr > 0.0 ? gapn / tr : (gapn == 0.0 ? 0.0 : INFINITY);
    converged = true_res <= tol;
    restart = gap >= RELIABLE_GAP || (recursive <= tol && !converged);
    if (io.verbose) std::printf(" %s reliable: true=%14.6E gap=%14.6E%s\n", name, true_res, gap, restart ? " RESTART" : "");
    return 0;
  }
};

#define CK(code)                         \
  do {                                   \
    if (c.err) return (code);            \
    if (check_launch(name)) return (code); \
  } while (0)
#define MV(in, out, code)            \
  do {                               \
    int _rc = c.mv((in), (out));     \
    if (_rc) return _rc;             \
  } while (0)

// QMRCCG with the FP64 recurrence scalars held on the GPU: one iteration is
// the p/q step, A p, the vt/wt step, A wt, one launch of the four inner
// products, the scalar recurrence in a single thread, the d/s/x/r step and
// |r|^2; the host waits once per iteration, for the residual it prints and
// tests (the reference waits for every inner-product group, cu:1079-1092).
// Same recurrence, reliable-residual checks, restart rule and MATVEC count as
// the reference (cu:434-443, cu:1071-1103).
struct DQState {
  double2 gamma, ksi, rho, eps, mu, tau, lambda, kappa, theta;
  // coefficients: p = co0 p + co1 vt, q = co2 q + co3 atw, vt = co4 vt + A p,
  // wt = co5 wt + q, d = co6 d + co7 p, s = co6 s + co7 A p
  double2 co[8];
  double bnorm, resid;
  int status, pad;
};

__host__ __device__ inline double2 dq_mul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__host__ __device__ inline double2 dq_div(double2 a, double2 b) {  // Smith's scaled complex division
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.y + b.x * r;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__host__ __device__ inline bool dq_zero(double2 a) { return a.x == 0.0 && a.y == 0.0; }
__host__ __device__ inline double2 dq_neg(double2 a) { return make_double2(-a.x, -a.y); }

// coefficients of the p/q and vt/wt steps from gamma, ksi, mu, tau
__host__ __device__ inline void dq_step_coefficients(DQState& S) {
  const double2 one = make_double2(1.0, 0.0);
  S.co[0] = dq_neg(S.mu);
  S.co[1] = dq_div(one, S.gamma);
  S.co[2] = dq_neg(dq_div(dq_mul(S.gamma, S.mu), S.ksi));
  S.co[3] = dq_div(one, S.ksi);
  S.co[4] = dq_neg(dq_div(S.tau, S.gamma));
  S.co[5] = dq_neg(dq_div(S.tau, S.ksi));
}

// the scalar recurrence of cu:442 from |vt|^2, |wt|^2, vt^T wt, vt^T A wt
__global__ void k_dq_recur(DQState* SP, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  DQState S = *SP;
  const double2 gamma0 = S.gamma, ksi0 = S.ksi, rho0 = S.rho, tau0 = S.tau, kappa0 = S.kappa;
  S.gamma = make_double2(sqrt(fmax(0.0, out[0].x)), 0.0);
  S.ksi = make_double2(sqrt(fmax(0.0, out[1].x)), 0.0);
  S.rho = out[2];
  S.eps = out[3];
  int st = 0;
  if (dq_zero(S.gamma)) st = 6;
  else if (dq_zero(S.ksi)) st = 7;
  const double2 den = dq_mul(dq_mul(S.gamma, S.tau), rho0);
  if (!st && dq_zero(den)) st = 12;
  if (!st) {
    S.mu = dq_div(dq_mul(dq_mul(gamma0, ksi0), S.rho), den);
    if (dq_zero(S.rho)) st = 13;
  }
  if (!st) {
    const double2 gm = dq_mul(S.gamma, S.mu), er = dq_div(S.eps, S.rho);
    S.tau = make_double2(er.x - gm.x, er.y - gm.y);
    const double at0 = tau0.x * tau0.x + tau0.y * tau0.y, ag = S.gamma.x * S.gamma.x + S.gamma.y * S.gamma.y;
    const double2 den2 = make_double2(S.lambda.x * at0 + ag, S.lambda.y * at0);
    if (dq_zero(den2)) st = 14;
    else {
      S.theta = dq_div(make_double2((1.0 - S.lambda.x) * at0, -S.lambda.y * at0), den2);
      const double2 g0t = dq_mul(gamma0, make_double2(tau0.x, -tau0.y));
      S.kappa = dq_neg(dq_div(dq_mul(g0t, kappa0), den2));
      S.lambda = dq_div(make_double2(S.lambda.x * at0, S.lambda.y * at0), den2);
    }
  }
  S.status = st;
  S.co[6] = S.theta;
  S.co[7] = S.kappa;
  if (!st) dq_step_coefficients(S);
  *SP = S;
}
__global__ void k_dq_resid(DQState* S, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double v = out[0].x;
  if (v < 0.0 && v > -1e-12) v = 0.0;
  S->resid = sqrt(v > 0.0 ? v : 0.0) / S->bnorm;
}

// d = zd d + za a (k_lincomb's arithmetic: zmulv per term, a zero zd drops d)
template <typename C> __device__ __forceinline__ C dq_lin(C d, double2 zd, C a, double2 za) {
  C v = mk<C>(0, 0);
  if (!dq_zero(zd)) v = zmulv(zd, d);
  return cadd(v, zmulv(za, a));
}
template <typename C>
__global__ void k_dq_pq(int n, C* p, C* q, const C* vt, const C* atw, const DQState* S) {
  const double2 c0 = S->co[0], c1 = S->co[1], c2 = S->co[2], c3 = S->co[3];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    p[i] = dq_lin(p[i], c0, vt[i], c1);
    q[i] = dq_lin(q[i], c2, atw[i], c3);
  }
}
template <typename C>
__global__ void k_dq_vw(int n, C* vt, C* wt, const C* ap, const C* q, const DQState* S) {
  const double2 c4 = S->co[4], c5 = S->co[5], one = make_double2(1.0, 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    vt[i] = dq_lin(vt[i], c4, ap[i], one);
    wt[i] = dq_lin(wt[i], c5, q[i], one);
  }
}
template <typename C>
__global__ void k_dq_dsxr(int n, C* d, C* s, C* x, C* r, const C* p, const C* ap, const DQState* S) {
  if (S->status) return;
  const double2 th = S->co[6], ka = S->co[7], one = make_double2(1.0, 0.0), mone = make_double2(-1.0, 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const C dn = dq_lin(d[i], th, p[i], ka);
    const C sn = dq_lin(s[i], th, ap[i], ka);
    d[i] = dn;
    s[i] = sn;
    x[i] = dq_lin(x[i], one, dn, one);
    r[i] = dq_lin(r[i], one, sn, mone);
  }
}

static inline unsigned dq_grid(int n) { return (unsigned)std::min<size_t>(ceil_div((size_t)std::max(n, 1), 256), 148 * 16); }

// ---------------------------------------------------------------- PBCGS2 (cu:459-480, cu:1168-1278)
// ZBCG2 = BiCGStab(2) with the reference's reliable updates and restarts, its
// FP64 scalars held on the GPU (DPState): the inner products land in device
// memory, single-thread kernels form rho/beta, sigma/alpha, the residual norm
// and the 3 x 3 minimal-residual step, and the vector updates read their
// coefficients from the state.  The host waits once per iteration (for the
// residual, the breakdown status and the reliable-update tests); the
// reference waits for every inner product (cu:1190-1255).
struct DPState {
  double2 alpha, omega, sigma, rho0, rho1, beta;
  double2 one, mone;
  double2 co[3];           // -beta, alpha, -alpha
  double2 y1, y2, my1, my2;  // Y1, Y2 of the minimal-residual step and their negatives
  double rnrm0, rnrm, mxnrmx, mxnrmr, resid;
  int status, xpdt, rcmp, pad;
};

__host__ __device__ inline double dp_abs(double2 a) { return hypot(a.x, a.y); }
__host__ __device__ inline double2 dp_conj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline double2 dp_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 dp_sc(double s, double2 a) { return make_double2(s * a.x, s * a.y); }

__global__ void k_dp_begin(DPState* S) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  S->rho0 = dq_neg(dq_mul(S->omega, S->rho0));
}
// rho1 = rr^H r_{k-1}, beta = alpha rho1 / rho0, rho0 = rho1
__global__ void k_dp_rho(DPState* S, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || S->status) return;
  S->rho1 = out[0];
  if (dq_zero(S->rho0)) { S->status = 95; return; }
  S->beta = dq_mul(S->alpha, dq_div(S->rho1, S->rho0));
  S->rho0 = S->rho1;
  S->co[0] = dq_neg(S->beta);
}
// sigma = rr^H u_k, alpha = rho1 / sigma
__global__ void k_dp_sigma(DPState* S, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || S->status) return;
  S->sigma = out[0];
  if (dq_zero(S->sigma)) { S->status = 98; return; }
  S->alpha = dq_div(S->rho1, S->sigma);
  S->co[1] = S->alpha;
  S->co[2] = dq_neg(S->alpha);
}
__global__ void k_dp_rnrm(DPState* S, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || S->status) return;
  S->rnrm = sqrt(fmax(0.0, out[0].x));
  S->mxnrmx = fmax(S->mxnrmx, S->rnrm);
  S->mxnrmr = fmax(S->mxnrmr, S->rnrm);
}
// the convex polynomial of cu:471-472 from the Gram matrix r_i^H r_j (lower
// triangle r0r0, r1r0, r1r1, r2r0, r2r1, r2r2 in out[0..5]) and the
// reliable-update tests of cu:474
__global__ void k_dp_gram(DPState* SP, const double2* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || SP->status) return;
  DPState S = *SP;
  double2 Zm[3][3];
  Zm[0][0] = out[0]; Zm[1][0] = out[1]; Zm[1][1] = out[2];
  Zm[2][0] = out[3]; Zm[2][1] = out[4]; Zm[2][2] = out[5];
  Zm[0][1] = dp_conj(Zm[1][0]); Zm[0][2] = dp_conj(Zm[2][0]); Zm[1][2] = dp_conj(Zm[2][1]);
  if (dq_zero(Zm[1][1])) { SP->status = 102; return; }
  double2 y0[3] = {make_double2(-1.0, 0.0), dq_div(Zm[1][0], Zm[1][1]), make_double2(0.0, 0.0)};
  double2 yl[3] = {make_double2(0.0, 0.0), dq_div(Zm[1][2], Zm[1][1]), make_double2(-1.0, 0.0)};
  auto matv = [&](const double2* v, double2* o) {
    for (int i = 0; i < 3; ++i) {
      o[i] = make_double2(0.0, 0.0);
      for (int j = 0; j < 3; ++j) o[i] = dp_add(o[i], dq_mul(Zm[i][j], v[j]));
    }
  };
  auto inner = [](const double2* a, const double2* b) {
    double2 sum = make_double2(0.0, 0.0);
    for (int i = 0; i < 3; ++i) sum = dp_add(sum, dq_mul(dp_conj(a[i]), b[i]));
    return sum;
  };
  double2 zy0[3], zyl[3];
  matv(y0, zy0);
  matv(yl, zyl);
  const double k0 = sqrt(dp_abs(inner(y0, zy0))), kl = sqrt(dp_abs(inner(yl, zyl)));
  if (k0 == 0.0 || kl == 0.0) { SP->status = 102; return; }
  const double2 vr = dp_sc(1.0 / (k0 * kl), inner(yl, zy0));
  const double avr = dp_abs(vr);
  if (avr == 0.0) { SP->status = 102; return; }
  const double2 fac = dp_sc((fmax(avr, 0.7) / avr) * (k0 / kl), vr);
  for (int i = 0; i < 3; ++i) y0[i] = make_double2(y0[i].x - dq_mul(fac, yl[i]).x, y0[i].y - dq_mul(fac, yl[i]).y);
  S.y1 = y0[1]; S.y2 = y0[2]; S.my1 = dq_neg(y0[1]); S.my2 = dq_neg(y0[2]);
  S.omega = y0[2];
  matv(y0, zy0);
  S.rnrm = sqrt(dp_abs(inner(y0, zy0)));
  S.mxnrmx = fmax(S.mxnrmx, S.rnrm);
  S.mxnrmr = fmax(S.mxnrmr, S.rnrm);
  const double delta = 1.0e-2;
  S.xpdt = S.rnrm < delta * S.rnrm0 && S.rnrm0 < S.mxnrmx;
  S.rcmp = (S.rnrm < delta * S.mxnrmr && S.rnrm0 < S.mxnrmr) || S.xpdt;
  S.resid = S.rnrm0 > 0.0 ? S.rnrm / S.rnrm0 : 0.0;
  *SP = S;
}
// d = cd d + ca a + cb b with coefficients read from device memory (null:
// term absent; a zero cd drops d), k_lincomb's arithmetic
template <typename C>
__global__ void k_dp_lin(int n, C* d, const double2* cd, const C* a, const double2* ca, const C* b,
                         const double2* cb, const int* status) {
  if (*status) return;
  const double2 zd = cd ? *cd : make_double2(0.0, 0.0), za = ca ? *ca : make_double2(0.0, 0.0),
                zb = cb ? *cb : make_double2(0.0, 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    C v = mk<C>(0, 0);
    if (!dq_zero(zd)) v = zmulv(zd, d[i]);
    if (a) v = cadd(v, zmulv(za, a[i]));
    if (b) v = cadd(v, zmulv(zb, b[i]));
    d[i] = v;
  }
}

template <typename T> int solve_pbcgs2(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "PBCGS2";
  Ctx<T> c(io, name);
  C *rr = c.w(0), *r[3] = {c.w(1), c.w(2), c.w(3)}, *u[3] = {c.w(4), c.w(5), c.w(6)};
  C *XP = c.w(7), *BP = c.w(8), *X = c.w(9);
  DPState* dS = nullptr;
  DPState* hS = nullptr;
  cudaEvent_t ev = nullptr;
  struct Free {
    DPState*& a; DPState*& b; cudaEvent_t& e;
    ~Free() { cudaFree(a); if (b) cudaFreeHost(b); if (e) cudaEventDestroy(e); }
  } release{dS, hS, ev};
  if (cudaMalloc((void**)&dS, sizeof(DPState)) != cudaSuccess || cudaMallocHost((void**)&hS, sizeof(DPState)) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    set_error(name, "scalar state allocation");
    return 29;
  }
  // init: rr=r0=BP=b, XP=x0, the rest 0 (cu:462)
  c.copy(XP, io.x);
  c.copy(rr, io.b); c.copy(r[0], io.b); c.copy(BP, io.b);
  c.zero(r[1]); c.zero(r[2]); c.zero(u[0]); c.zero(u[1]); c.zero(u[2]); c.zero(X);
  const double rnrm0 = c.nrm(r[0]);
  CK(92);
  DPState S{};
  S.alpha = make_double2(0.0, 0.0); S.omega = make_double2(1.0, 0.0); S.sigma = make_double2(1.0, 0.0);
  S.rho0 = make_double2(1.0, 0.0); S.rho1 = make_double2(0.0, 0.0);
  S.one = make_double2(1.0, 0.0); S.mone = make_double2(-1.0, 0.0);
  S.rnrm0 = rnrm0; S.rnrm = S.mxnrmx = S.mxnrmr = rnrm0;
  S.resid = rnrm0 > 0.0 ? 1.0 : 0.0;
  auto upload = [&]() -> int {
    *hS = S;
    if (cudaMemcpyAsync(dS, hS, sizeof(DPState), cudaMemcpyHostToDevice, c.st()) != cudaSuccess ||
        cudaStreamSynchronize(c.st()) != cudaSuccess) {
      set_error(name, "scalar state upload");
      return 1;
    }
    return 0;
  };
  if (upload()) return 93;
  double resid = S.resid;
  const int n = c.n;
  const unsigned gb = dq_grid(n);
  const int* dst = &dS->status;
  auto lin = [&](C* d, const double2* cd, const C* a, const double2* ca, const C* b = nullptr,
                 const double2* cb = nullptr) {
    k_dp_lin<C><<<gb, 256, 0, c.st()>>>(n, d, cd, a, ca, b, cb, dst);
    note_launch();
  };
  const double2 *one = &dS->one, *mbeta = &dS->co[0], *calpha = &dS->co[1], *cmalpha = &dS->co[2];
  int it = 0;
  while (resid > io.tol && it < io.maxit) {
    ++it;
    k_dp_begin<<<1, 32, 0, c.st()>>>(dS);
    note_launch();
    for (int k = 1; k <= 2; ++k) {
      {
        const C* A1[1] = {rr};
        const C* B1[1] = {r[k - 1]};
        const int cj[1] = {1};
        if (io.ops->dots_dev(n, 1, A1, B1, cj)) return 94;
      }
      k_dp_rho<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
      note_launch();
      for (int j = 0; j < k; ++j) lin(u[j], mbeta, r[j], one);  // u_j = r_j - beta u_j
      MV(u[k - 1], u[k], 96);
      {
        const C* A1[1] = {rr};
        const C* B1[1] = {u[k]};
        const int cj[1] = {1};
        if (io.ops->dots_dev(n, 1, A1, B1, cj)) return 97;
      }
      k_dp_sigma<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
      note_launch();
      lin(X, one, u[0], calpha);                                                  // X += alpha u0
      for (int j = 0; j < k; ++j) lin(r[j], one, u[j + 1], cmalpha);              // r_j -= alpha u_{j+1}
      MV(r[k - 1], r[k], 99);
      {
        const C* A1[1] = {r[0]};
        const int cj[1] = {1};
        if (io.ops->dots_dev(n, 1, A1, A1, cj)) return 100;
      }
      k_dp_rnrm<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
      note_launch();
    }
    {  // Hermitian Gram matrix r_i^H r_j, lower triangle (cu:1215-1220)
      const C* A6[6] = {r[0], r[1], r[1], r[2], r[2], r[2]};
      const C* B6[6] = {r[0], r[0], r[1], r[0], r[1], r[2]};
      const int cj[6] = {1, 1, 1, 1, 1, 1};
      if (io.ops->dots_dev(n, 6, A6, B6, cj)) return 101;
    }
    k_dp_gram<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
    note_launch();
    // u0 -= Y1 u1 + Y2 u2 ; X += Y1 r0 + Y2 r1 ; r0 -= Y1 r1 + Y2 r2
    lin(u[0], one, u[1], &dS->my1, u[2], &dS->my2);
    lin(X, one, r[0], &dS->y1, r[1], &dS->y2);
    lin(r[0], one, r[1], &dS->my1, r[2], &dS->my2);
    if (check_launch(name)) return 103;
    if (cudaMemcpyAsync(hS, dS, sizeof(DPState), cudaMemcpyDeviceToHost, c.st()) != cudaSuccess ||
        cudaEventRecord(ev, c.st()) != cudaSuccess || cudaEventSynchronize(ev) != cudaSuccess) {
      set_error(name, "scalar state read-back");
      return 103;
    }
    S = *hS;
    if (S.status == 95) { set_error(name, "ZBCG2 breakdown: RHO0 == 0"); return 95; }
    if (S.status == 98) { set_error(name, "ZBCG2 breakdown: SIGMA == 0"); return 98; }
    if (S.status == 102) { set_error(name, "ZBCG2 convex-polynomial breakdown"); return 102; }
    resid = S.resid;
    bool changed = false;
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      int rc = c.reliable("PBCGS2", BP, X, r[0], rnrm0, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 104 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(r[0], BP, io.sy);        // r0 = BP - A X
        c.lin(XP, 1.0, X, 1.0);          // XP += X
        c.zero(X);
        c.copy(BP, r[0]);
        c.copy(rr, r[0]);
        c.zero(r[1]); c.zero(r[2]); c.zero(u[0]); c.zero(u[1]); c.zero(u[2]);
        S.rnrm = S.mxnrmx = S.mxnrmr = tres * rnrm0;
        S.alpha = make_double2(0.0, 0.0); S.omega = make_double2(1.0, 0.0); S.sigma = make_double2(1.0, 0.0);
        S.rho0 = make_double2(1.0, 0.0);
        resid = S.resid = tres;
        CK(104);
        if (upload()) return 104;
        if (io.verbose) std::printf(" PBCGS2 reliable restart at iteration %d\n", it);
        continue;
      }
    }
    if (S.rcmp) {
      MV(X, io.sy, 104);
      c.diff(r[0], BP, io.sy);
      if (S.xpdt) {
        c.lin(XP, 1.0, X, 1.0);
        c.zero(X);
        c.copy(BP, r[0]);
      }
      S.mxnrmr = S.rnrm;
      if (S.xpdt) S.mxnrmx = S.rnrm;
      CK(104);
      changed = true;
    }
    if (changed && upload()) return 104;
    if (io.verbose) std::printf(" PBCGS2 iteration=%6d residual=%14.6E\n", it, resid);
  }
  // X = X + XP and one final true residual against the original b (cu:1259-1264)
  c.lin(X, 1.0, XP, 1.0);
  MV(X, io.sy, 105);
  c.diff(r[0], io.b, io.sy);
  const double rnrm = c.nrm(r[0]);
  CK(106);
  resid = rnrm0 > 0.0 ? rnrm / rnrm0 : INFINITY;
  c.copy(io.x, X);
  CK(107);
  io.itno = it; io.tole = resid; io.ncompte = c.nc;
  return 0;  // ZBCG2 reports non-convergence through TOLE only (cu:1275-1277)
}

// ---------------------------------------------------------------- QMRCCG (cu:434-443, cu:1071-1103)
template <typename T> int solve_qmrccg(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "QMRCCG";
  Ctx<T> c(io, name);
  C *r = c.w(0), *p = c.w(1), *ap = c.w(2), *q = c.w(3), *d = c.w(4), *s = c.w(5);
  C *vt = c.w(6), *wt = c.w(7), *atw = c.w(8), *xs = c.w(9);
  const double bnorm = c.nrm(io.b);
  CK(52);
  if (bnorm == 0.0) { set_error(name, "zero RHS norm"); return 52; }
  DQState* dS = nullptr;
  DQState* hS = nullptr;
  cudaEvent_t ev = nullptr;
  struct Free {
    DQState*& a; DQState*& b; cudaEvent_t& e;
    ~Free() { cudaFree(a); if (b) cudaFreeHost(b); if (e) cudaEventDestroy(e); }
  } release{dS, hS, ev};
  if (cudaMalloc((void**)&dS, sizeof(DQState)) != cudaSuccess || cudaMallocHost((void**)&hS, sizeof(DQState)) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    set_error(name, "scalar state allocation");
    return 29;
  }
  c.copy(xs, io.x);
  MV(xs, io.sy, 53);
  c.diff(r, io.b, io.sy);
  c.zero(p); c.zero(ap); c.zero(q); c.zero(d); c.zero(s); c.zero(atw);
  c.copy(vt, r); c.copy(wt, r);
  DQState S{};
  S.bnorm = bnorm;
  // initial scalars (host, as at every restart), then uploaded with the step coefficients
  auto init_scalars = [&]() -> int {
    const C* A3[3] = {vt, wt, vt};
    const C* B3[3] = {vt, wt, wt};
    const int cj[3] = {1, 1, 0};
    double2 o[3];
    if (io.ops->dots(c.n, 3, A3, B3, cj, o)) return 54;
    const double gn = std::sqrt(std::max(0.0, o[0].x)), kn = std::sqrt(std::max(0.0, o[1].x));
    const double2 rho = o[2];
    int rc = c.mv(wt, atw);
    if (rc) return rc;
    const double2 eps = dz(c.dotu(vt, atw));
    if (c.err) return 54;
    if (dq_zero(rho) || gn == 0.0 || kn == 0.0) {
      char msg[80];
      std::snprintf(msg, sizeof(msg), "breakdown at step %d", dq_zero(rho) ? 5 : (gn == 0.0 ? 6 : 7));
      set_error(name, msg);
      return 55;
    }
    S.lambda = make_double2(1.0, 0.0); S.kappa = make_double2(-1.0, 0.0); S.theta = make_double2(-1.0, 0.0);
    S.gamma = make_double2(gn, 0.0); S.ksi = make_double2(kn, 0.0); S.mu = make_double2(0.0, 0.0);
    S.rho = rho; S.eps = eps;
    S.tau = dq_div(eps, rho);
    S.status = 0;
    dq_step_coefficients(S);
    *hS = S;
    if (cudaMemcpyAsync(dS, hS, sizeof(DQState), cudaMemcpyHostToDevice, c.st()) != cudaSuccess ||
        cudaStreamSynchronize(c.st()) != cudaSuccess) {
      set_error(name, "scalar state upload");
      return 54;
    }
    return 0;
  };
  int rc = init_scalars();
  if (rc) return rc;
  double resid = c.nrm(r) / bnorm;
  CK(55);
  const int n = c.n;
  const unsigned gb = dq_grid(n);
  int it = 0;
  while (it < io.maxit && resid > io.tol) {
    ++it;
    k_dq_pq<C><<<gb, 256, 0, c.st()>>>(n, p, q, vt, atw, dS);
    note_launch();
    MV(p, ap, 56);
    k_dq_vw<C><<<gb, 256, 0, c.st()>>>(n, vt, wt, ap, q, dS);
    note_launch();
    MV(wt, atw, 57);
    {
      const C* A4[4] = {vt, wt, vt, vt};
      const C* B4[4] = {vt, wt, wt, atw};
      const int cj[4] = {1, 1, 0, 0};
      if (io.ops->dots_dev(n, 4, A4, B4, cj)) return 57;
    }
    k_dq_recur<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
    note_launch();
    k_dq_dsxr<C><<<gb, 256, 0, c.st()>>>(n, d, s, xs, r, p, ap, dS);
    note_launch();
    {
      const C* A1[1] = {r};
      const int cj[1] = {1};
      if (io.ops->dots_dev(n, 1, A1, A1, cj)) return 59;
    }
    k_dq_resid<<<1, 32, 0, c.st()>>>(dS, io.ops->d_out);
    note_launch();
    if (check_launch(name)) return 59;
    if (cudaMemcpyAsync(hS, dS, sizeof(DQState), cudaMemcpyDeviceToHost, c.st()) != cudaSuccess ||
        cudaEventRecord(ev, c.st()) != cudaSuccess || cudaEventSynchronize(ev) != cudaSuccess) {
      set_error(name, "scalar state read-back");
      return 59;
    }
    if (hS->status) {
      char msg[80];
      std::snprintf(msg, sizeof(msg), "breakdown at step %d", hS->status);
      set_error(name, msg);
      return 58;
    }
    resid = hS->resid;
    if (io.verbose) std::printf(" QMRCCG iteration=%6d residual=%14.6E\n", it, resid);
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      rc = c.reliable("QMRCCG", io.b, xs, r, bnorm, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 59 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(io.sy, io.b, io.sy);
        c.copy(r, io.sy);
        c.zero(p); c.zero(ap); c.zero(q); c.zero(d); c.zero(s); c.zero(atw);
        c.copy(vt, io.sy); c.copy(wt, io.sy);
        if ((rc = init_scalars())) return rc;
        resid = tres;
      }
    }
  }
  if (resid > io.tol) {
    double tres;
    bool conv, rest;
    rc = c.reliable("QMRCCG", io.b, xs, r, bnorm, resid, io.tol, tres, conv, rest);
    if (rc) return rc == 1 ? 60 : rc;
    resid = tres;
  }
  c.copy(io.x, xs);
  CK(61);
  io.itno = it; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

// ---------------------------------------------------------------- PBCGST (cu:445-457, cu:1105-1165)
template <typename T> int solve_pbcgst(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "PBCGST";
  Ctx<T> c(io, name);
  C *r = c.w(0), *rt = c.w(1), *p = c.w(2), *sv = c.w(3), *v = c.w(4), *t = c.w(5), *xs = c.w(6), *rtrue = c.w(7);
  const Engine<T>& E = *io.eng;
  const C* adia_full = io.adia_full ? io.adia_full : io.adia;  // the DIAGL preconditioner reads the full layout
  auto precon = [&](C* dst, const C* src) { v_precon<T>(dst, src, adia_full, E.occ, E.g.nat, E.g.nat0, c.st()); };
  c.copy(xs, io.x);
  const double bnorm = c.nrm(io.b);
  CK(72);
  int total_it = 0, restart = 0;
  double resid = 1.0;
  bool converged = false;
  while (total_it < io.maxit && !converged) {
    if (restart > 0 && io.verbose) std::printf(" restart PBCGST CUDA: %d\n", restart);
    MV(xs, io.sy, 73);
    c.diff(rtrue, io.b, io.sy);
    precon(r, rtrue);
    c.copy(rt, r);
    c.zero(p);
    c.zero(v);
    Z rho = 1.0, alpha = 1.0, omega = 1.0;
    for (int local = 0; local < 5 && total_it < io.maxit && !converged; ++local) {
      const Z new_rho = c.dotc(rt, r);
      CK(74);
      const Z kap = rho * omega;
      if (kap == Z(0.0)) { set_error(name, "hard breakdown at step 6 (rho0*omega == 0)"); return 75; }
      const Z beta = new_rho * alpha / kap;
      rho = new_rho;
      // p = r + beta (p - omega v)
      c.lin(p, beta, v, -beta * omega);
      c.lin(p, 1.0, r, 1.0);
      MV(p, io.sy, 76);
      precon(v, io.sy);
      const Z xi = c.dotc(rt, v);
      CK(77);
      if (xi == Z(0.0)) { set_error(name, "hard breakdown at step 10 (rtilde^H v == 0)"); return 78; }
      alpha = rho / xi;
      c.copy(sv, r);
      c.lin(sv, 1.0, v, -alpha);
      const double snorm = c.nrm(sv);
      CK(79);
      if (snorm < 1.19209e-7) {  // PIM step 12 soft breakdown: accept x += alpha p, restart
        c.lin(xs, 1.0, p, alpha);
        ++total_it;
        if (io.verbose) std::printf(" PBCGST CUDA soft breakdown: restarting from updated x at iteration %d\n", total_it);
        break;
      }
      MV(sv, io.sy, 80);
      precon(t, io.sy);
      Z tt, ts;
      {
        const C* A2[2] = {t, t};
        const C* B2[2] = {t, sv};
        const int cj[2] = {1, 1};
        double2 o[2];
        if (io.ops->dots(c.n, 2, A2, B2, cj, o)) return 81;
        tt = zd(o[0]);
        ts = zd(o[1]);
      }
      if (tt == Z(0.0)) { set_error(name, "hard breakdown at step 14 (t^H t == 0)"); return 82; }
      omega = ts / tt;
      c.lin(xs, 1.0, p, alpha, sv, omega);
      c.copy(r, sv);
      c.lin(r, 1.0, t, -omega);
      ++total_it;
      MV(xs, io.sy, 84);
      c.diff(rtrue, io.b, io.sy);
      const double trn = c.nrm(rtrue);
      CK(84);
      resid = bnorm > 0.0 ? trn / bnorm : INFINITY;
      if (io.verbose) std::printf(" PBCGST iteration=%6d residual=%14.6E\n", total_it, resid);
      if (resid <= io.tol) converged = true;
    }
    ++restart;
  }
  if (!converged) {
    MV(xs, io.sy, 85);
    c.diff(rtrue, io.b, io.sy);
    const double trn = c.nrm(rtrue);
    CK(85);
    resid = bnorm > 0.0 ? trn / bnorm : INFINITY;
  }
  c.copy(io.x, xs);
  CK(86);
  io.itno = total_it; io.tole = resid; io.ncompte = c.nc;
  if (!converged) { set_error(name, "MAXIT reached before requested tolerance"); return 87; }
  return 0;
}

// ---------------------------------------------------------------- PETRKP (cu:482-493, cu:1280-1357)
template <typename T> int solve_petrkp(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "PETRKP";
  Ctx<T> c(io, name);
  C *ace = c.w(0), *gi = c.w(1), *pi = c.w(2), *qi = c.w(3), *axi = c.w(4), *rv = c.w(5), *xs = c.w(6);
  c.copy(xs, io.x);
  const double bb = c.dotc(io.b, io.b).real();
  CK(112);
  {
    int rc = c.mv(io.b, io.sy, 1);  // ACE = A^H b
    if (rc) return rc;
  }
  c.copy(ace, io.sy); c.copy(gi, io.sy); c.copy(pi, io.sy);
  MV(pi, io.sy, 113);
  c.copy(qi, io.sy);
  double gg = c.dotc(gi, gi).real(), qq = c.dotc(qi, qi).real();
  CK(114);
  if (qq == 0.0) { set_error(name, "breakdown: ||QI|| == 0 while computing initial alpha"); return 115; }
  double alpha = gg / qq;
  c.lin(xs, 1.0, pi, alpha);
  MV(xs, io.sy, 116);
  c.copy(axi, io.sy);
  double resid = 1.0;
  int it;
  for (it = 1; it <= io.maxit; ++it) {
    const double oldgg = gg;
    {
      int rc = c.mv(axi, io.sy, 1);  // A^H A x
      if (rc) return rc;
    }
    c.diff(gi, ace, io.sy);
    gg = c.dotc(gi, gi).real();
    CK(118);
    if (oldgg == 0.0) { set_error(name, "breakdown: previous ||GI|| == 0 while computing beta"); return 119; }
    const double beta = gg / oldgg;
    c.lin(pi, beta, gi, 1.0);
    MV(pi, io.sy, 120);
    c.copy(qi, io.sy);
    qq = c.dotc(qi, qi).real();
    CK(120);
    if (qq == 0.0) { set_error(name, "breakdown: ||QI|| == 0 while computing alpha"); return 121; }
    alpha = gg / qq;
    c.lin(xs, 1.0, pi, alpha);
    if (it != 10 * (it / 10)) {
      c.lin(axi, 1.0, qi, alpha);
    } else {
      MV(xs, io.sy, 122);
      c.copy(axi, io.sy);
    }
    c.diff(rv, axi, io.b);
    const double rr = c.dotc(rv, rv).real();
    CK(123);
    resid = bb > 0.0 ? std::sqrt(std::max(rr, 0.0) / bb) : INFINITY;
    if (io.verbose) std::printf(" PETRKP iteration=%6d residual=%14.6E\n", it, resid);
    if (resid < io.tol) break;
  }
  c.copy(io.x, xs);
  CK(124);
  io.itno = it <= io.maxit ? it : io.maxit; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

// ---------------------------------------------------------------- GPBICG (cu:420-432, cu:1031-1069)
template <typename T> int solve_gpbicg(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "GPBICG";
  Ctx<T> c(io, name);
  C *r0 = c.w(0), *p = c.w(1), *r = c.w(2), *yv = c.w(3), *t = c.w(4), *ap = c.w(5), *at = c.w(6);
  C *u = c.w(7), *wv = c.w(8), *zv = c.w(9), *xsol = c.w(10), *told = c.w(11), *tmp = c.w(12);
  c.copy(xsol, io.x);
  const double bnorm = c.nrm(io.b);
  CK(32);
  if (bnorm == 0.0) { set_error(name, "zero RHS norm"); return 32; }
  MV(xsol, io.sy, 32);
  c.diff(r0, io.b, io.sy);
  c.copy(r, r0);
  c.zero(p); c.zero(t); c.zero(u); c.zero(wv); c.zero(zv); c.zero(yv); c.zero(told);
  Z r0rn = c.dotc(r0, r0), beta = 0.0, alpha = 0.0, dzeta = 0.0, eta = 0.0;
  double resid = c.nrm(r) / bnorm;
  CK(32);
  int it = 0;
  bool first = true;
  while (it < io.maxit && resid > io.tol) {
    ++it;
    // p = r + beta (p - u)
    c.lin(p, beta, u, -beta);
    c.lin(p, 1.0, r, 1.0);
    MV(p, io.sy, 33);
    c.copy(ap, io.sy);
    const Z g0 = c.dotc(r0, ap);
    CK(34);
    if (g0 == Z(0.0)) { set_error(name, "alpha breakdown"); return 34; }
    alpha = r0rn / g0;
    // y = (t - r) + alpha (ap - w) ; told = t ; t = r - alpha ap
    c.copy(yv, t);
    c.lin(yv, 1.0, r, -1.0);
    c.lin(yv, 1.0, ap, alpha, wv, -alpha);
    c.copy(told, t);
    c.copy(t, r);
    c.lin(t, 1.0, ap, -alpha);
    MV(t, io.sy, 35);
    c.copy(at, io.sy);
    Z g1, g4;
    {
      const C* A2[2] = {at, at};
      const C* B2[2] = {at, t};
      const int cj[2] = {1, 1};
      double2 o[2];
      if (io.ops->dots(c.n, 2, A2, B2, cj, o)) return 35;
      g1 = zd(o[0]);
      g4 = zd(o[1]);
    }
    if (first) {
      if (g1 == Z(0.0)) { set_error(name, "dzeta/eta breakdown"); return 36; }
      eta = 0.0;
      dzeta = g4 / g1;
    } else {
      const C* A3[3] = {yv, at, yv};
      const C* B3[3] = {yv, yv, t};
      const int cj[3] = {1, 1, 1};
      double2 o[3];
      if (io.ops->dots(c.n, 3, A3, B3, cj, o)) return 35;
      const Z g2 = zd(o[0]), g3 = zd(o[1]), g5 = zd(o[2]);
      const Z den = g1 * g2 - g3 * std::conj(g3);
      if (den == Z(0.0)) { set_error(name, "dzeta/eta breakdown"); return 36; }
      dzeta = (g2 * g4 - g5 * g3) / den;
      eta = (g1 * g5 - std::conj(g3) * g4) / den;
    }
    // u = dz ap + eta (told - r + beta u) ; z = dz r + eta z - alpha u ; x += alpha p + z ; r = t - eta y - dz at
    c.copy(tmp, told);
    c.lin(tmp, 1.0, r, -1.0);
    c.lin(tmp, 1.0, u, beta);
    c.lin(u, 0.0, ap, dzeta, tmp, eta);
    c.lin(zv, eta, r, dzeta, u, -alpha);
    c.lin(xsol, 1.0, p, alpha, zv, 1.0);
    c.copy(r, t);
    c.lin(r, 1.0, yv, -eta, at, -dzeta);
    resid = c.nrm(r) / bnorm;
    CK(37);
    if (io.verbose) std::printf(" GPBICG iteration=%6d residual=%14.6E\n", it, resid);
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      int rc = c.reliable("GPBICG", io.b, xsol, r, bnorm, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 37 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(io.sy, io.b, io.sy);
        c.copy(r0, io.sy); c.copy(r, io.sy);
        c.zero(p); c.zero(yv); c.zero(t); c.zero(ap); c.zero(at); c.zero(u); c.zero(wv); c.zero(zv); c.zero(told);
        r0rn = c.dotc(r0, r0);
        CK(37);
        beta = 0.0;
        first = true;
        resid = tres;
        continue;
      }
    }
    const Z g0b = c.dotc(r0, r);
    CK(39);
    if (r0rn == Z(0.0) || dzeta == Z(0.0)) { set_error(name, "beta breakdown"); return 39; }
    beta = (alpha * g0b / dzeta) / r0rn;
    r0rn = g0b;
    c.lin(wv, 0.0, at, 1.0, ap, beta);
    first = false;
  }
  if (resid > io.tol) {
    double tres;
    bool conv, rest;
    int rc = c.reliable("GPBICG", io.b, xsol, r, bnorm, resid, io.tol, tres, conv, rest);
    if (rc) return rc == 1 ? 40 : rc;
    resid = tres;
  }
  c.copy(io.x, xsol);
  CK(40);
  io.itno = it; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

// ---------------------------------------------------------------- BiCGStab(4) (cu:1363-1433)
template <typename T> int solve_bicgstab4(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "BiCGStab4";
  Ctx<T> c(io, name);
  C* r[5] = {c.w(0), c.w(3), c.w(4), c.w(5), c.w(6)};
  C* u[5] = {c.w(1), c.w(7), c.w(8), c.w(9), c.w(10)};
  C* rtil = c.w(2);
  C* x = io.x;
  MV(x, io.sy, 132);
  c.diff(r[0], io.b, io.sy);
  const double bnorm = c.nrm(io.b);
  double rnorm = c.nrm(r[0]);
  CK(132);
  if (bnorm == 0.0) { set_error(name, "zero RHS norm"); return 133; }
  double resid = rnorm / bnorm;
  if (resid <= io.tol) { io.itno = 0; io.tole = resid; io.ncompte = c.nc; return 0; }
  if (rnorm < 1e-30) { set_error(name, "cannot start from zero residual"); return 133; }
  c.lin(rtil, 0.0, r[0], 1.0 / rnorm);
  c.zero(u[0]);
  Z rho = 1.0, alpha = 0.0, omega = 1.0;
  int it;
  for (it = 1; it <= io.maxit; ++it) {
    rho = -omega * rho;
    for (int j = 0; j < 4; ++j) {
      if (std::abs(rho) < 1e-30) { set_error(name, "breakdown: rho is zero"); return 135; }
      const Z rho1 = c.dotc(rtil, r[j]);
      CK(135);
      const Z beta = alpha * rho1 / rho;
      rho = rho1;
      for (int i = 0; i <= j; ++i) c.lin(u[i], -beta, r[i], 1.0);
      MV(u[j], u[j + 1], 136);
      const Z den = c.dotc(rtil, u[j + 1]);
      CK(137);
      if (std::abs(den) < 1e-30) { set_error(name, "breakdown: <rtilde,u> is zero"); return 137; }
      alpha = rho / den;
      for (int i = 0; i <= j; ++i) c.lin(r[i], 1.0, u[i + 1], -alpha);
      MV(r[j], r[j + 1], 138);
      c.lin(x, 1.0, u[0], alpha);
    }
    Z tau[4][4], gp[5], gam[5], gpp[5];
    double sigma[5] = {0, 0, 0, 0, 0};
    for (auto& row : tau) for (auto& zz : row) zz = 0.0;
    for (int i = 0; i < 5; ++i) gp[i] = gam[i] = gpp[i] = 0.0;
    for (int j = 1; j <= 4; ++j) {
      for (int i = 1; i < j; ++i) {
        const Z dd = c.dotc(r[i], r[j]);
        CK(140);
        tau[j - 1][i - 1] = dd / sigma[i];
        c.lin(r[j], 1.0, r[i], -tau[j - 1][i - 1]);
      }
      sigma[j] = c.dotc(r[j], r[j]).real();
      CK(141);
      if (!(sigma[j] > 1e-30)) { set_error(name, "breakdown in MR polynomial"); return 141; }
      gp[j] = c.dotc(r[j], r[0]) / sigma[j];
      CK(141);
    }
    omega = gam[4] = gp[4];
    for (int j = 3; j >= 1; --j) {
      gam[j] = gp[j];
      for (int i = j + 1; i <= 4; ++i) gam[j] -= tau[i - 1][j - 1] * gam[i];
    }
    for (int j = 1; j < 4; ++j) {
      gpp[j] = gam[j + 1];
      for (int i = j + 1; i < 4; ++i) gpp[j] += tau[i - 1][j - 1] * gam[i + 1];
    }
    c.lin(x, 1.0, r[0], gam[1]);
    c.lin(r[0], 1.0, r[4], -gp[4]);
    c.lin(u[0], 1.0, u[4], -gam[4]);
    for (int j = 1; j < 4; ++j) {
      c.lin(x, 1.0, r[j], gpp[j]);
      c.lin(r[0], 1.0, r[j], -gp[j]);
      c.lin(u[0], 1.0, u[j], -gam[j]);
    }
    rnorm = c.nrm(r[0]);
    CK(143);
    resid = rnorm / bnorm;
    if (io.verbose) std::printf(" BiCGStab(4) iteration=%6d residual=%14.6E\n", it, resid);
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      int rc = c.reliable("BiCGStab(4)", io.b, x, r[0], bnorm, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 144 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(r[0], io.b, io.sy);
        rnorm = tres * bnorm;
        if (!(rnorm > 0.0)) { set_error(name, "reliable restart produced zero residual"); return 144; }
        c.lin(rtil, 0.0, r[0], 1.0 / rnorm);
        c.zero(u[0]);
        rho = 1.0; alpha = 0.0; omega = 1.0;
        resid = tres;
      }
    }
  }
  MV(x, io.sy, 144);
  c.diff(r[0], io.b, io.sy);
  rnorm = c.nrm(r[0]);
  CK(144);
  resid = rnorm / bnorm;
  io.itno = it <= io.maxit ? it : io.maxit; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

// Gaussian elimination with partial pivoting and the 1e-30 breakdown test of cu:349-359
static bool solve_small(Z* a, Z* b, int n, int ld) {
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = std::abs(a[k * ld + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = std::abs(a[i * ld + k]);
      if (v > best) { best = v; piv = i; }
    }
    if (best < 1e-30) return false;
    if (piv != k) {
      for (int j = k; j < n; ++j) std::swap(a[k * ld + j], a[piv * ld + j]);
      std::swap(b[k], b[piv]);
    }
    for (int i = k + 1; i < n; ++i) {
      const Z f = a[i * ld + k] / a[k * ld + k];
      a[i * ld + k] = 0.0;
      for (int j = k + 1; j < n; ++j) a[i * ld + j] -= f * a[k * ld + j];
      b[i] -= f * b[k];
    }
  }
  for (int i = n - 1; i >= 0; --i) {
    Z v = b[i];
    for (int j = i + 1; j < n; ++j) v -= a[i * ld + j] * b[j];
    if (std::abs(a[i * ld + i]) < 1e-30) return false;
    b[i] = v / a[i * ld + i];
  }
  return true;
}

// ---------------------------------------------------------------- GPBiCGStab(2) (cu:1435-1491)
template <typename T> int solve_gpbicgstab2(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "GPBiCGStab2";
  Ctx<T> c(io, name);
  C *r0 = c.w(0), *p0 = c.w(1), *rt = c.w(2), *z = c.w(3), *yv = c.w(4), *u = c.w(5), *hs = c.w(6), *hq0 = c.w(7),
    *hq1 = c.w(8), *work = c.w(9);
  C* x = io.x;
  MV(x, io.sy, 152);
  c.diff(r0, io.b, io.sy);
  const double bnorm = c.nrm(io.b);
  double rnorm = c.nrm(r0);
  CK(152);
  if (bnorm == 0.0) { set_error(name, "zero RHS norm"); return 153; }
  c.copy(rt, r0); c.copy(p0, r0); c.zero(z);
  bool fresh = true;
  double resid = rnorm / bnorm;
  Z rho, sigma, alpha, beta;
  int it;
  for (it = 1; it <= io.maxit && resid > io.tol; ++it) {
    if (fresh) {
      rho = c.dotc(rt, r0);
      MV(p0, work, 154);
      sigma = c.dotc(rt, work);
      CK(154);
      if (std::abs(sigma) < 1e-30) { set_error("GP2", "sigma1 zero"); return 154; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha);
      c.lin(r0, 1.0, work, -alpha);
      MV(r0, hs, 155);
      rho = c.dotc(rt, hs);
      CK(155);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0);
      c.lin(work, -beta, hs, 1.0);
      MV(work, hq1, 156);
      sigma = c.dotc(rt, hq1);
      CK(156);
      if (std::abs(sigma) < 1e-30) { set_error("GP2", "sigma2 zero"); return 156; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha);
      c.lin(r0, 1.0, work, -alpha);
      c.lin(hs, 1.0, hq1, -alpha);
      MV(hs, hq0, 157);
      rho = c.dotc(rt, hq0);
      CK(157);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0);
      c.lin(work, -beta, hs, 1.0);
      c.lin(hq1, -beta, hq0, 1.0);
      Z mat[3][3], rhs[3];
      mat[0][0] = c.dotc(hs, hs); mat[0][1] = c.dotc(hs, hq0); mat[1][1] = c.dotc(hq0, hq0);
      rhs[0] = c.dotc(hs, r0); rhs[1] = c.dotc(hq0, r0);
      CK(159);
      mat[1][0] = std::conj(mat[0][1]);
      if (!solve_small(&mat[0][0], rhs, 2, 3)) { set_error("GP2", "initial 2x2 minimization breakdown"); return 159; }
      const Z z1 = rhs[0], z2 = rhs[1];
      c.lin(z, 0.0, r0, z1, hs, z2);
      c.lin(x, 1.0, z, 1.0);
      c.lin(yv, 0.0, hs, z1, hq0, z2);
      c.lin(u, 0.0, work, z1, hq1, z2);
      c.lin(r0, 1.0, yv, -1.0);
      c.lin(p0, 1.0, u, -1.0);
      c.copy(hq0, work);
      fresh = false;
    } else {
      rho = c.dotc(rt, r0);
      MV(p0, work, 161);
      sigma = c.dotc(rt, work);
      CK(161);
      if (std::abs(sigma) < 1e-30) { set_error("GP2", "sigma1 zero"); return 161; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha);
      c.lin(z, 1.0, u, -alpha);
      c.lin(yv, 1.0, hq0, -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha);
      c.lin(hs, 1.0, hq1, -alpha);
      MV(r0, hq1, 162);
      rho = c.dotc(rt, hq1);
      CK(162);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0);
      c.lin(work, -beta, hq1, 1.0);
      c.lin(hq0, -beta, hs, 1.0);
      c.lin(u, -beta, yv, 1.0);
      MV(work, hs, 163);
      sigma = c.dotc(rt, hs);
      CK(163);
      if (std::abs(sigma) < 1e-30) { set_error("GP2", "sigma2 zero"); return 163; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha);
      c.lin(z, 1.0, u, -alpha);
      c.lin(yv, 1.0, hq0, -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha);
      c.lin(hq1, 1.0, hs, -alpha);
      MV(hq1, hq0, 164);
      rho = c.dotc(rt, hq0);
      CK(164);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0);
      c.lin(work, -beta, hq1, 1.0);
      c.lin(hs, -beta, hq0, 1.0);
      c.lin(u, -beta, yv, 1.0);
      Z mat[3][3], rhs[3];
      {
        const C* A9[8] = {hq1, hq1, hq1, hq0, hq0, yv, hq1, hq0};
        const C* B9[8] = {hq1, hq0, yv, hq0, yv, yv, r0, r0};
        const int cj[8] = {1, 1, 1, 1, 1, 1, 1, 1};
        double2 o[8];
        if (io.ops->dots(c.n, 8, A9, B9, cj, o)) return 166;
        mat[0][0] = zd(o[0]); mat[0][1] = zd(o[1]); mat[0][2] = zd(o[2]);
        mat[1][1] = zd(o[3]); mat[1][2] = zd(o[4]); mat[2][2] = zd(o[5]);
        rhs[0] = zd(o[6]); rhs[1] = zd(o[7]);
        rhs[2] = c.dotc(yv, r0);
        CK(166);
      }
      mat[1][0] = std::conj(mat[0][1]); mat[2][0] = std::conj(mat[0][2]); mat[2][1] = std::conj(mat[1][2]);
      if (!solve_small(&mat[0][0], rhs, 3, 3)) { set_error("GP2", "3x3 minimization breakdown"); return 166; }
      const Z z1 = rhs[0], z2 = rhs[1], eta = rhs[2];
      c.lin(z, eta, r0, z1, hq1, z2);
      c.lin(x, 1.0, z, 1.0);
      c.lin(yv, eta, hq1, z1, hq0, z2);
      c.lin(u, eta, work, z1, hs, z2);
      c.lin(r0, 1.0, yv, -1.0);
      c.lin(p0, 1.0, u, -1.0);
      // restore fixed histories: hs=r1, hq0=p1, hq1=p2 (cu:1474)
      c.copy(hq0, hs);
      c.copy(hs, hq1);
      c.copy(hq1, hq0);
      c.copy(hq0, work);
    }
    rnorm = c.nrm(r0);
    CK(169);
    resid = rnorm / bnorm;
    if (io.verbose) std::printf(" GPBiCGStab(2) iteration=%6d residual=%14.6E\n", it, resid);
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      int rc = c.reliable("GPBiCGStab(2)", io.b, x, r0, bnorm, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 170 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(r0, io.b, io.sy);
        c.copy(rt, r0); c.copy(p0, r0); c.zero(z);
        fresh = true;
        resid = tres;
      }
    }
  }
  if (resid > io.tol) {
    MV(x, io.sy, 172);
    c.diff(r0, io.b, io.sy);
    rnorm = c.nrm(r0);
    CK(172);
    resid = rnorm / bnorm;
  }
  io.itno = it <= io.maxit ? it : io.maxit; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

// ---------------------------------------------------------------- GPBiCGStab(4) (cu:1493-1570)
template <typename T> int solve_gpbicgstab4(SolveIO<T>& io) {
  using C = cplx<T>;
  const char* name = "GPBiCGStab4";
  Ctx<T> c(io, name);
  C *r0 = c.w(0), *p0 = c.w(1), *rt = c.w(2), *z = c.w(3), *yv = c.w(4), *u = c.w(5);
  C* hs[3] = {c.w(6), c.w(7), c.w(8)};
  C* hq[4] = {c.w(9), c.w(10), c.w(11), c.w(12)};
  C* work = io.sy;  // the MATVEC staging vector doubles as `work`, as in the reference
  C* x = io.x;
  MV(x, io.sy, 182);
  c.diff(r0, io.b, io.sy);
  const double bnorm = c.nrm(io.b);
  double rnorm = c.nrm(r0);
  CK(182);
  if (bnorm == 0.0) { set_error("GP4", "zero RHS norm"); return 183; }
  c.copy(rt, r0); c.copy(p0, r0); c.zero(z);
  bool fresh = true;
  double resid = rnorm / bnorm;
  Z rho, sigma, alpha, beta, zeta[4], eta;
  auto restore = [&]() {
    c.copy(hq[0], hs[0]); c.copy(hs[0], hq[3]); c.copy(hq[3], hq[0]);
    c.copy(hq[0], hs[1]); c.copy(hs[1], hq[2]); c.copy(hq[2], hq[0]);
    c.copy(hq[0], hs[2]); c.copy(hs[2], hq[1]); c.copy(hq[1], hq[0]); c.copy(hq[0], work);
  };
  auto gram = [&](C* const* rr, int with_y, Z* mat, Z* rhs, int ld) -> int {
    for (int i = 0; i < 4; ++i) {
      for (int j = 0; j < 4; ++j) mat[i * ld + j] = c.dotc(rr[i + 1], rr[j + 1]);
      if (with_y) {
        mat[i * ld + 4] = c.dotc(rr[i + 1], yv);
        mat[4 * ld + i] = std::conj(mat[i * ld + 4]);
      }
      rhs[i] = c.dotc(rr[i + 1], rr[0]);
    }
    if (with_y) {
      mat[4 * ld + 4] = c.dotc(yv, yv);
      rhs[4] = c.dotc(yv, rr[0]);
    }
    return c.err;
  };
  int it;
  for (it = 1; it <= io.maxit && resid > io.tol; ++it) {
    if (fresh) {
      C* rr[5] = {r0, hq[3], hq[2], hq[1], hq[0]};
      C* pp[5] = {p0, work, hs[2], hs[1], hs[0]};
      rho = c.dotc(rt, rr[0]);
      CK(184);
      for (int j = 1; j <= 4; ++j) {
        MV(pp[j - 1], pp[j], 184);
        sigma = c.dotc(rt, pp[j]);
        CK(184);
        if (std::abs(sigma) < 1e-30) { set_error("GP4", "initial sigma zero"); return 184; }
        alpha = rho / sigma;
        c.lin(x, 1.0, pp[0], alpha);
        for (int i = 0; i < j; ++i) c.lin(rr[i], 1.0, pp[i + 1], -alpha);
        MV(rr[j - 1], rr[j], 185);
        rho = c.dotc(rt, rr[j]);
        CK(185);
        beta = rho / sigma;
        for (int i = 0; i <= j; ++i) c.lin(pp[i], -beta, rr[i], 1.0);
      }
      Z mat[5][5], rhs[5];
      for (auto& row : mat) for (auto& v : row) v = 0.0;
      for (auto& v : rhs) v = 0.0;
      if (gram(rr, 0, &mat[0][0], rhs, 5)) return 187;
      if (!solve_small(&mat[0][0], rhs, 4, 5)) { set_error("GP4", "initial 4x4 minimization breakdown"); return 187; }
      for (int i = 0; i < 4; ++i) zeta[i] = rhs[i];
      c.lin(z, 0.0, rr[0], zeta[0]);
      for (int i = 1; i < 4; ++i) c.lin(z, 1.0, rr[i], zeta[i]);
      c.lin(x, 1.0, z, 1.0);
      c.lin(yv, 0.0, rr[1], zeta[0]);
      c.lin(u, 0.0, pp[1], zeta[0]);
      for (int i = 1; i < 4; ++i) { c.lin(yv, 1.0, rr[i + 1], zeta[i]); c.lin(u, 1.0, pp[i + 1], zeta[i]); }
      c.lin(r0, 1.0, yv, -1.0);
      c.lin(p0, 1.0, u, -1.0);
      restore();
      fresh = false;
    } else {
      rho = c.dotc(rt, r0);
      // j = 1
      MV(p0, work, 190);
      sigma = c.dotc(rt, work);
      CK(190);
      if (std::abs(sigma) < 1e-30) { set_error("GP4", "sigma1 zero"); return 190; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha); c.lin(z, 1.0, u, -alpha); c.lin(yv, 1.0, hq[0], -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha);
      for (int i = 0; i < 3; ++i) c.lin(hs[i], 1.0, hq[i + 1], -alpha);
      MV(r0, hq[3], 191);
      rho = c.dotc(rt, hq[3]);
      CK(191);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0); c.lin(work, -beta, hq[3], 1.0);
      for (int i = 0; i < 3; ++i) c.lin(hq[i], -beta, hs[i], 1.0);
      c.lin(u, -beta, yv, 1.0);
      // j = 2
      MV(work, hs[2], 193);
      sigma = c.dotc(rt, hs[2]);
      CK(193);
      if (std::abs(sigma) < 1e-30) { set_error("GP4", "sigma2 zero"); return 193; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha); c.lin(z, 1.0, u, -alpha); c.lin(yv, 1.0, hq[0], -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha); c.lin(hq[3], 1.0, hs[2], -alpha);
      for (int i = 0; i < 2; ++i) c.lin(hs[i], 1.0, hq[i + 1], -alpha);
      MV(hq[3], hq[2], 194);
      rho = c.dotc(rt, hq[2]);
      CK(194);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0); c.lin(work, -beta, hq[3], 1.0); c.lin(hs[2], -beta, hq[2], 1.0);
      for (int i = 0; i < 2; ++i) c.lin(hq[i], -beta, hs[i], 1.0);
      c.lin(u, -beta, yv, 1.0);
      // j = 3
      MV(hs[2], hs[1], 196);
      sigma = c.dotc(rt, hs[1]);
      CK(196);
      if (std::abs(sigma) < 1e-30) { set_error("GP4", "sigma3 zero"); return 196; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha); c.lin(z, 1.0, u, -alpha); c.lin(yv, 1.0, hq[0], -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha); c.lin(hq[3], 1.0, hs[2], -alpha); c.lin(hq[2], 1.0, hs[1], -alpha);
      c.lin(hs[0], 1.0, hq[1], -alpha);
      MV(hq[2], hq[1], 197);
      rho = c.dotc(rt, hq[1]);
      CK(197);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0); c.lin(work, -beta, hq[3], 1.0); c.lin(hs[2], -beta, hq[2], 1.0);
      c.lin(hs[1], -beta, hq[1], 1.0); c.lin(hq[0], -beta, hs[0], 1.0); c.lin(u, -beta, yv, 1.0);
      // j = 4
      MV(hs[1], hs[0], 199);
      sigma = c.dotc(rt, hs[0]);
      CK(199);
      if (std::abs(sigma) < 1e-30) { set_error("GP4", "sigma4 zero"); return 199; }
      alpha = rho / sigma;
      c.lin(x, 1.0, p0, alpha); c.lin(z, 1.0, u, -alpha); c.lin(yv, 1.0, hq[0], -alpha, work, alpha);
      c.lin(r0, 1.0, work, -alpha); c.lin(hq[3], 1.0, hs[2], -alpha); c.lin(hq[2], 1.0, hs[1], -alpha);
      c.lin(hq[1], 1.0, hs[0], -alpha);
      MV(hq[1], hq[0], 200);
      rho = c.dotc(rt, hq[0]);
      CK(200);
      beta = rho / sigma;
      c.lin(p0, -beta, r0, 1.0); c.lin(work, -beta, hq[3], 1.0); c.lin(hs[2], -beta, hq[2], 1.0);
      c.lin(hs[1], -beta, hq[1], 1.0); c.lin(hs[0], -beta, hq[0], 1.0); c.lin(u, -beta, yv, 1.0);
      C* rr[5] = {r0, hq[3], hq[2], hq[1], hq[0]};
      C* pp[5] = {p0, work, hs[2], hs[1], hs[0]};
      Z mat[5][5], rhs[5];
      for (auto& row : mat) for (auto& v : row) v = 0.0;
      for (auto& v : rhs) v = 0.0;
      if (gram(rr, 1, &mat[0][0], rhs, 5)) return 202;
      if (!solve_small(&mat[0][0], rhs, 5, 5)) { set_error("GP4", "5x5 minimization breakdown"); return 202; }
      for (int i = 0; i < 4; ++i) zeta[i] = rhs[i];
      eta = rhs[4];
      c.lin(z, eta);
      for (int i = 0; i < 4; ++i) c.lin(z, 1.0, rr[i], zeta[i]);
      c.lin(x, 1.0, z, 1.0);
      c.lin(yv, eta);
      c.lin(u, eta);
      for (int i = 0; i < 4; ++i) { c.lin(yv, 1.0, rr[i + 1], zeta[i]); c.lin(u, 1.0, pp[i + 1], zeta[i]); }
      c.lin(r0, 1.0, yv, -1.0);
      c.lin(p0, 1.0, u, -1.0);
      restore();
    }
    rnorm = c.nrm(r0);
    CK(205);
    resid = rnorm / bnorm;
    if (io.verbose) std::printf(" GPBiCGStab(4) iteration=%6d residual=%14.6E\n", it, resid);
    if ((it % RELIABLE_PERIOD) == 0 || resid <= io.tol) {
      double tres;
      bool conv, rest;
      int rc = c.reliable("GPBiCGStab(4)", io.b, x, r0, bnorm, resid, io.tol, tres, conv, rest);
      if (rc) return rc == 1 ? 206 : rc;
      if (conv) { resid = tres; break; }
      if (rest) {
        c.diff(r0, io.b, io.sy);
        c.copy(rt, r0); c.copy(p0, r0); c.zero(z);
        fresh = true;
        resid = tres;
      } else {
        c.copy(work, hq[0]);  // the check overwrote `work` (the MATVEC staging vector)
      }
    }
  }
  MV(x, io.sy, 206);
  c.diff(r0, io.b, io.sy);
  rnorm = c.nrm(r0);
  CK(206);
  resid = rnorm / bnorm;
  io.itno = it <= io.maxit ? it : io.maxit; io.tole = resid; io.ncompte = c.nc;
  return 0;
}

#define DDB_SOLVERS(T)                                   \
  template int solve_pbcgs2<T>(SolveIO<T>&);             \
  template int solve_qmrccg<T>(SolveIO<T>&);             \
  template int solve_pbcgst<T>(SolveIO<T>&);             \
  template int solve_petrkp<T>(SolveIO<T>&);             \
  template int solve_gpbicg<T>(SolveIO<T>&);             \
  template int solve_bicgstab4<T>(SolveIO<T>&);          \
  template int solve_gpbicgstab2<T>(SolveIO<T>&);        \
  template int solve_gpbicgstab4<T>(SolveIO<T>&);
DDB_SOLVERS(float)
DDB_SOLVERS(double)
#undef DDB_SOLVERS

}  // namespace ddb
