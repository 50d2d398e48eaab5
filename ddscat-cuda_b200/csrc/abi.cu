// C ABI of the B200 DDA library: the 15 entry points of
// ddscat_cuda_unified/cuda/ddscat_matvec_cuda.h:11-51 with the reference's
// argument checks, return codes, last_error() text convention and state
// lifetime (device state owned from prepare until release or the next
// prepare; the solution stays resident for EVALQ/SCAT).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>
#include <mutex>
#include <thread>
#include "ddscat_b200.h"
#include "batch.h"
#include "solvers.h"

namespace ddb {

// error text of the calling host thread (the multi-target solve runs targets
// on several threads; single-threaded callers see the reference behaviour)
static thread_local std::string g_last_error;
void set_error(const char* where, const char* what) {
  char b[1024];
  std::snprintf(b, sizeof(b), "%s: %s", where, what);
  g_last_error = b;
}
void set_cuda_error(const char* where, cudaError_t e) { set_error(where, cudaGetErrorString(e)); }
const char* last_error_text() { return g_last_error.c_str(); }
void clear_error() { g_last_error.clear(); }
static std::atomic<unsigned long long> g_launches{0};
void note_launch(unsigned long long k) { g_launches += k; }
unsigned long long launch_total() { return g_launches.load(); }
bool env_flag(const char* name) {
  const char* v = std::getenv(name);
  return v && *v && !(v[0] == '0' && v[1] == '\0');
}
// raise the dynamic shared-memory limit of kernel f once per process (thread-safe)
void raise_smem_limit(const void* f) {
  static std::mutex mu;
  static std::vector<const void*> done;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), f) != done.end()) return;
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  done.push_back(f);
}
int check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { set_cuda_error(where, e); return 1; }
  return 0;
}

using C = float2;

struct State {
  bool ready = false;
  bool solution_valid = false;
  Engine<float> eng;
  VecOps<float> ops;
  cudaStream_t stream = 0;
  C *d_xf = nullptr, *d_yf = nullptr, *d_adia = nullptr, *d_aoff = nullptr;  // full 3*NAT
  C *d_b = nullptr, *d_sx = nullptr, *d_sy = nullptr, *d_work = nullptr;     // compact
  C *d_adia_c = nullptr, *d_aoff_c = nullptr;  // compact CXADIA / CXAOFF of the current solve
  bool aoff_zero = false;
  // how the target was prepared (for the all-FP64 engine built on demand)
  int prep_kind = 0;  // 1 prepare_green, 2 prepare (CPU Green)
  GreenArgs<float> green_args;
  std::vector<float2> cpu_green;  // CXZC copy for prepare_f32
  int16_t* h_iocc = nullptr;
  int device = -1;  // the CUDA device current at prepare, which holds the state's buffers
};
static State s;

// batched-solve buffers and statistics (library extension)
struct BatchState {
  int R = 0, cap = 0, n = 0;
  C *b = nullptr, *x = nullptr, *adia = nullptr, *aoff = nullptr, *work = nullptr;
  BatchOps<float> ops;
  double matvec_ms = 0.0;
  long long matvec_rhs = 0;
  int matvec_calls = 0;
};
static BatchState bs;
static void release_batch() {
  cudaFree(bs.b); cudaFree(bs.x); cudaFree(bs.adia); cudaFree(bs.aoff); cudaFree(bs.work);
  bs.ops.release();
  const double ms = bs.matvec_ms;
  const long long mr = bs.matvec_rhs;
  const int mc = bs.matvec_calls;
  bs = BatchState{};
  bs.matvec_ms = ms; bs.matvec_rhs = mr; bs.matvec_calls = mc;
}

// all-FP64 engine of the prepared target (FP64 true residuals / FP64 solves)
struct F64State {
  bool ready = false;
  Engine<double> eng;
  VecOps<double> ops;
  double2 *x = nullptr, *y = nullptr, *b = nullptr, *ad = nullptr, *ao = nullptr;
};
static F64State f64;
static void release_f64() {
  if (f64.ready) {
    cudaFree(f64.x); cudaFree(f64.y); cudaFree(f64.b); cudaFree(f64.ad); cudaFree(f64.ao);
    f64.ops.release();
    f64.eng.release();
  }
  f64 = F64State{};
}

// all-FP64 batched solve (complex128 vectors, FP64 engine)
struct Batch64 {
  int R = 0, cap = 0, n = 0;
  double2 *b = nullptr, *x = nullptr, *adia = nullptr, *aoff = nullptr, *work = nullptr, *full = nullptr;
  BatchOps<double> ops;
};
static Batch64 b64;
static void release_b64() {
  cudaFree(b64.b); cudaFree(b64.x); cudaFree(b64.adia); cudaFree(b64.aoff); cudaFree(b64.work); cudaFree(b64.full);
  b64.ops.release();
  b64 = Batch64{};
}

static void release_state() {
  release_batch();
  release_b64();
  release_f64();
  delete[] s.h_iocc;
  s.h_iocc = nullptr;
  if (s.ready || s.eng.green) {
    cudaFree(s.d_xf); cudaFree(s.d_yf); cudaFree(s.d_adia); cudaFree(s.d_aoff);
    cudaFree(s.d_b); cudaFree(s.d_sx); cudaFree(s.d_sy); cudaFree(s.d_work);
    cudaFree(s.d_adia_c); cudaFree(s.d_aoff_c);
    s.ops.release();
    s.eng.release();
  }
  s.cpu_green.clear();
  s = State{};
}

// Console output level.  1 (the default, as the reference prints for DDSCAT
// users): the per-MATVEC and per-iteration lines of the 15 reference entry
// points (cu:417, e.g. cu:1085-1092); 0: silent; 2: also the library
// extensions' diagnostics (batched-solve phase times, multi-target set-up).
// DDSCAT_B200_VERBOSE=0/1/2 sets it; ddscat_b200_set_verbose overrides it.
static int g_verbose = -1;
int verbose_level() {
  if (g_verbose >= 0) return g_verbose;
  const char* v = std::getenv("DDSCAT_B200_VERBOSE");
  if (!v || !*v) return 1;
  const int l = std::atoi(v);
  return l < 0 ? 0 : (l > 2 ? 2 : l);
}

static int slices_build() {
#ifdef DDSCAT_B200_SLICES
  return 1;
#else
  return 0;
#endif
}

static int allocate_runtime() {
  const size_t n = (size_t)3 * s.eng.g.nat, cn = (size_t)3 * s.eng.g.nat0;
  if (cn > (size_t)0x7fffffff) { set_error("allocate runtime", "3*NAT0 exceeds solver int range"); return 204; }
  cudaError_t e = cudaSuccess;
  auto M = [&](C** p, size_t cnt) { if (e == cudaSuccess) e = cudaMalloc((void**)p, cnt * sizeof(C)); };
  M(&s.d_xf, n); M(&s.d_yf, n); M(&s.d_adia, n); M(&s.d_aoff, n);
  M(&s.d_b, cn); M(&s.d_sx, cn); M(&s.d_sy, cn); M(&s.d_work, 13 * cn);
  M(&s.d_adia_c, cn); M(&s.d_aoff_c, cn);
  if (e != cudaSuccess) { set_cuda_error("allocate runtime", e); return 204; }
  if (s.ops.init(s.stream)) return 204;
  s.eng.stream = s.stream;
  s.eng.slices_layout = slices_build();
  if (s.eng.ensure_workspace(1)) return 204;
  return 0;
}

// True when every byte of the host array is zero: 64-bit words, large arrays
// split over up to 8 host threads (a full DDSCAT vector at 128^3 is 50 MB).
static bool zero_words(const unsigned char* c, size_t bytes) {
  size_t i = 0;
  for (; i < bytes && ((uintptr_t)(c + i) & 7u); ++i)
    if (c[i]) return false;
  const uint64_t* w = reinterpret_cast<const uint64_t*>(c + i);
  const size_t nw = (bytes - i) / 8;
  for (size_t k = 0; k < nw; k += 64) {
    uint64_t acc = 0;
    const size_t e = std::min(nw, k + 64);
    for (size_t j = k; j < e; ++j) acc |= w[j];
    if (acc) return false;
  }
  for (i += nw * 8; i < bytes; ++i)
    if (c[i]) return false;
  return true;
}
static bool all_zero(const void* p, size_t bytes) {
  const unsigned char* c = (const unsigned char*)p;
  const size_t part = (size_t)8 << 20;
  const int nt = (int)std::min<size_t>(8, (bytes + part - 1) / part);
  if (nt <= 1) return zero_words(c, bytes);
  std::vector<std::thread> th;
  std::vector<char> res(nt, 0);
  const size_t chunk = (bytes + nt - 1) / nt;
  for (int k = 0; k < nt; ++k) {
    const size_t off = (size_t)k * chunk, len = std::min(chunk, bytes - std::min(bytes, off));
    th.emplace_back([&, k, off, len]() { res[k] = zero_words(c + off, len) ? 1 : 0; });
  }
  for (auto& t : th) t.join();
  for (char r : res)
    if (!r) return false;
  return true;
}

// ---- copies of the caller's pageable host arrays ----
// DDSCAT passes pageable Fortran arrays (a full vector is 50 MB at 128^3).  A
// pageable cudaMemcpy is staged by the driver at a few GB/s; here the host side
// of the staging is split over up to 8 threads into two pinned 8 MB buffers
// that alternate with their DMA on the library stream.  Same semantics as the
// synchronous copy for the caller: its array is read (or written) completely
// before the call returns.
constexpr size_t PIN_CHUNK = (size_t)8 << 20;
struct PinnedStage {
  char* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool ok = false, tried = false;
};
static PinnedStage g_pin;

static void par_copy(void* dst, const void* src, size_t bytes) {
  const int nt = (int)std::min<size_t>(8, bytes >> 20);
  if (nt <= 1) { std::memcpy(dst, src, bytes); return; }
  const size_t ch = (bytes + nt - 1) / nt;
  std::vector<std::thread> th;
  for (int k = 0; k < nt; ++k) {
    const size_t off = (size_t)k * ch, len = std::min(ch, bytes - std::min(bytes, off));
    if (len) th.emplace_back([=]() { std::memcpy((char*)dst + off, (const char*)src + off, len); });
  }
  for (auto& t : th) t.join();
}

static bool pin_ready() {
  if (g_pin.tried) return g_pin.ok;
  g_pin.tried = true;
  bool ok = true;
  for (int k = 0; k < 2 && ok; ++k)
    ok = cudaMallocHost((void**)&g_pin.buf[k], PIN_CHUNK) == cudaSuccess &&
         cudaEventCreateWithFlags(&g_pin.ev[k], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) cudaGetLastError();  // fall back to pageable copies
  g_pin.ok = ok;
  return ok;
}

static cudaError_t copy_h2d(void* dev, const void* host, size_t bytes) {
  if (bytes < 2 * PIN_CHUNK || !pin_ready()) return cudaMemcpy(dev, host, bytes, cudaMemcpyHostToDevice);
  cudaError_t e = cudaSuccess;
  int k = 0;
  for (size_t off = 0; off < bytes && e == cudaSuccess; off += PIN_CHUNK, k ^= 1) {
    const size_t n = std::min(PIN_CHUNK, bytes - off);
    e = cudaEventSynchronize(g_pin.ev[k]);  // the DMA that last read buf[k] has finished
    if (e != cudaSuccess) break;
    par_copy(g_pin.buf[k], (const char*)host + off, n);
    e = cudaMemcpyAsync((char*)dev + off, g_pin.buf[k], n, cudaMemcpyHostToDevice, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(g_pin.ev[k], s.stream);
  }
  return e;
}

static cudaError_t copy_d2h(void* host, const void* dev, size_t bytes) {
  if (bytes < 2 * PIN_CHUNK || !pin_ready()) return cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost);
  const size_t nch = (bytes + PIN_CHUNK - 1) / PIN_CHUNK;
  auto issue = [&](size_t i) {
    const size_t off = i * PIN_CHUNK, n = std::min(PIN_CHUNK, bytes - off);
    cudaError_t e = cudaMemcpyAsync(g_pin.buf[i & 1], (const char*)dev + off, n, cudaMemcpyDeviceToHost, s.stream);
    return e == cudaSuccess ? cudaEventRecord(g_pin.ev[i & 1], s.stream) : e;
  };
  cudaError_t e = issue(0);
  for (size_t i = 0; i < nch && e == cudaSuccess; ++i) {
    if (i + 1 < nch) e = issue(i + 1);  // buf[(i+1)&1] was drained to the host in round i-1
    if (e == cudaSuccess) e = cudaEventSynchronize(g_pin.ev[i & 1]);
    if (e != cudaSuccess) break;
    const size_t off = i * PIN_CHUNK;
    par_copy((char*)host + off, g_pin.buf[i & 1], std::min(PIN_CHUNK, bytes - off));
  }
  return e;
}

static int upload_operators(const void* adia, const void* aoff) {
  const size_t b = (size_t)3 * s.eng.g.nat * sizeof(C);
  // zero CXAOFF (isotropic materials) contributes nothing: neither copied nor read
  s.aoff_zero = all_zero(aoff, b);
  cudaError_t e = copy_h2d(s.d_adia, adia, b);
  if (e == cudaSuccess && !s.aoff_zero) e = copy_h2d(s.d_aoff, aoff, b);
  if (e != cudaSuccess) { set_cuda_error("operator H2D", e); return 1; }
  return 0;
}

// maybe_zero: the array may be all zero (an initial guess): then the compact
// vector is cleared on the device instead of copied
static int upload_full_to_compact(const void* host, C* compact, bool maybe_zero = false) {
  const size_t b = (size_t)3 * s.eng.g.nat * sizeof(C);
  if (maybe_zero && all_zero(host, b)) {
    const cudaError_t z = cudaMemsetAsync(compact, 0, (size_t)3 * s.eng.g.nat0 * sizeof(C), s.stream);
    if (z != cudaSuccess) { set_cuda_error("zero initial guess", z); return 1; }
    return 0;
  }
  cudaError_t e = copy_h2d(s.d_xf, host, b);
  if (e != cudaSuccess) { set_cuda_error("full vector H2D", e); return 1; }
  v_gather<float>(s.d_xf, compact, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  return check_launch("full->compact gather");
}

static int download_compact_to_full(const C* compact, void* host) {
  const size_t b = (size_t)3 * s.eng.g.nat * sizeof(C);
  cudaError_t e = cudaMemsetAsync(s.d_xf, 0, b, s.stream);
  if (e != cudaSuccess) { set_cuda_error("solution compact D2H", e); return 1; }
  v_scatter<float>(compact, s.d_xf, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  if (check_launch("compact->full scatter")) return 1;
  e = copy_d2h(host, s.d_xf, b);
  if (e != cudaSuccess) { set_cuda_error("solution compact D2H", e); return 1; }
  return 0;
}

typedef int (*SolveFn)(SolveIO<float>&);

struct SolverCodes {
  const char* name;
  int invalid, workspace, h2d, d2h;
  bool publish_on_maxit;  // PBCGST writes x back before returning 87
};

static int run_solver(const SolverCodes& sc, SolveFn fn, const void* b, void* x, const void* adia, const void* aoff,
                      int ndim, int maxit, float tol, int* itout, float* tole, int* ncout) {
  clear_error();
  if (!s.ready || !b || !x || !adia || !aoff || !itout || !tole || !ncout || ndim != 3 * s.eng.g.nat || maxit <= 0 ||
      tol <= 0.f) {
    set_error(sc.name, "invalid argument");
    return sc.invalid;
  }
  if (!s.d_work) { set_error(sc.name, "Krylov workspace missing"); return sc.workspace; }
  s.solution_valid = false;
  if (upload_full_to_compact(b, s.d_b)) return sc.h2d;
  if (upload_full_to_compact(x, s.d_sx, true)) return sc.h2d;
  if (upload_operators(adia, aoff)) return sc.h2d;
  // the MATVEC's finish reads CXADIA / CXAOFF in the layout of x: compact
  // copies let it stage them with x in shared memory
  v_gather<float>(s.d_adia, s.d_adia_c, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  if (!s.aoff_zero) v_gather<float>(s.d_aoff, s.d_aoff_c, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  if (check_launch("CXADIA/CXAOFF gather")) return sc.h2d;
  SolveIO<float> io;
  io.eng = &s.eng; io.ops = &s.ops; io.stream = s.stream;
  io.n = 3 * s.eng.g.nat0;
  io.b = s.d_b; io.x = s.d_sx;
  io.adia = s.d_adia_c; io.aoff = s.aoff_zero ? nullptr : s.d_aoff_c; io.a_full = 0;
  io.adia_full = s.d_adia;
  io.work = s.d_work; io.sy = s.d_sy;
  io.maxit = maxit; io.tol = (double)tol; io.verbose = verbose_level() >= 1;
  int rc = fn(io);
  if (io.verbose) std::fflush(stdout);
  if (rc == 0 || (rc == 87 && sc.publish_on_maxit)) {
    const int mc = matvec_check(s.eng);
    if (mc) return mc;
  }
  if (rc != 0 && !(rc == 87 && sc.publish_on_maxit)) return rc;
  std::string keep = g_last_error;
  if (download_compact_to_full(s.d_sx, x)) return sc.d2h;
  s.solution_valid = true;
  *itout = io.itno;
  *tole = (float)io.tole;
  *ncout = io.ncompte;
  if (rc) g_last_error = keep;
  return rc;
}

// ---- far-field quadrature (cu:849-875) ----
struct IntDir {
  float k[3];
  double w[5];
};
static long lround_half_away(double v) { return v >= 0 ? (long)std::floor(v + 0.5) : -(long)std::floor(-v + 0.5); }
static int make_integration_dirs(const float ak[3], const C e01[3], float etasca, int nat0, std::vector<IntDir>& dirs) {
  const double pi = 4.0 * std::atan(1.0);
  const double ak2 = (double)ak[0] * ak[0] + (double)ak[1] * ak[1] + (double)ak[2] * ak[2], akk = std::sqrt(ak2);
  double a1[3] = {(double)e01[0].x, (double)e01[1].x, (double)e01[2].x};
  const double einc = std::sqrt(a1[0] * a1[0] + a1[1] * a1[1] + a1[2] * a1[2]);
  if (!(einc > 0.0)) { set_error("GPU SCAT", "CXE01_TF is pure imaginary"); return 1; }
  for (double& v : a1) v *= akk / einc;
  const double a2[3] = {(ak[1] * a1[2] - ak[2] * a1[1]) / akk, (ak[2] * a1[0] - ak[0] * a1[2]) / akk,
                        (ak[0] * a1[1] - ak[1] * a1[0]) / akk};
  const double x = akk * std::cbrt(3.0 * (double)nat0 / (4.0 * pi)), theta0 = 2.0 * pi / (1.0 + x), afac = 1.0;
  const int ntheta = 1 + (int)lround_half_away((2.0 * (3.0 + x) / (double)etasca) * (1.0 + afac / (pi + theta0)) /
                                               (1.0 + afac * theta0 / ((pi + theta0) * (pi + theta0))));
  double theta = 0.0, thetau = 0.0;
  dirs.clear();
  for (int ic = 1; ic <= ntheta; ++ic) {
    const double thetal = theta;
    theta = thetau;
    if (ic < ntheta) {
      const double si = (double)ic * (pi + afac * pi / (theta0 + pi)) / (double)(ntheta - 1), term = si - afac - theta0;
      thetau = 0.5 * (term + std::sqrt(term * term + 4.0 * theta0 * si));
    } else {
      thetau = pi;
    }
    const double domega = 2.0 * pi * (std::cos(0.5 * (thetal + theta)) - std::cos(0.5 * (theta + thetau)));
    const double ct = std::cos(theta), st = std::sin(theta), ct2 = ct * ct;
    int nphi = (ic == 1 || ic == ntheta) ? 1 : (int)lround_half_away(4.0 * pi * st / (thetau - thetal));
    if (nphi < 3 && ic != 1 && ic != ntheta) nphi = 3;
    const double w = domega / (double)nphi, dphi = 2.0 * pi / (double)nphi;
    for (int ip = 1; ip <= nphi; ++ip) {
      const double phi = dphi * ((double)ip - 0.5 * (double)(ic % 2)), sp = std::sin(phi), cp = std::cos(phi);
      IntDir d{};
      for (int k = 0; k < 3; ++k) d.k[k] = (float)(ct * (double)ak[k] + st * (cp * a1[k] + sp * a2[k]));
      d.w[0] = w; d.w[1] = w * ct; d.w[2] = w * st * cp; d.w[3] = w * st * sp; d.w[4] = w * ct2;
      dirs.push_back(d);
    }
  }
  return 0;
}

// Csca, Csca*g (3), Csca*<cos^2>, and the backscatter term (last direction)
// from the far-field sums F(n) = sum_j P_j exp(-i k_s . r_j) at the
// integration directions: |F - n (n . F)|^2 weighted by the quadrature
// (ddscat_matvec_cuda.cu:975-1002), times |k|^4 / E02.
static void scat_integrate(const std::vector<IntDir>& dirs, const double2* sums, double ak2, double e02,
                           double* cbksca, double* csca, double* cscag, double* cscag2) {
  const double akk = std::sqrt(ak2);
  const int nd = (int)dirs.size();
  double acc[5] = {0, 0, 0, 0, 0}, back = 0.0;
  for (int i = 0; i < nd; ++i) {
    const double nx = dirs[i].k[0] / akk, ny = dirs[i].k[1] / akk, nz = dirs[i].k[2] / akk;
    const double2 sx = sums[3 * i], sy = sums[3 * i + 1], sz = sums[3 * i + 2];
    const double ndr = nx * sx.x + ny * sy.x + nz * sz.x, ndi = nx * sx.y + ny * sy.y + nz * sz.y;
    const double exr = sx.x - nx * ndr, exi = sx.y - nx * ndi, eyr = sy.x - ny * ndr, eyi = sy.y - ny * ndi;
    const double ezr = sz.x - nz * ndr, ezi = sz.y - nz * ndi;
    const double es2 = exr * exr + exi * exi + eyr * eyr + eyi * eyi + ezr * ezr + ezi * ezi;
    for (int k = 0; k < 5; ++k) acc[k] += es2 * dirs[i].w[k];
    if (i == nd - 1) back = es2;
  }
  const double fac = ak2 * ak2 / e02;
  *csca = fac * acc[0];
  cscag[0] = fac * acc[1];
  cscag[1] = fac * acc[2];
  cscag[2] = fac * acc[3];
  *cscag2 = fac * acc[4];
  *cbksca = fac * back;
}

// ---- batched solve ----
static bool is_device_ptr(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int ensure_batch(int R) {
  const int n = 3 * s.eng.g.nat0;
  if (bs.n == n && bs.cap >= R && bs.work) {  // reuse the vectors; reductions sized for R
    if (bs.R != R) {
      bs.ops.release();
      if (bs.ops.init(R, n, s.stream)) return 1;
      bs.R = R;
    }
    return 0;
  }
  release_batch();
  const size_t v = (size_t)R * n;
  cudaError_t e = cudaMalloc((void**)&bs.b, v * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&bs.x, v * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&bs.adia, v * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&bs.aoff, v * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&bs.work, (size_t)BATCH_WORK_VECTORS * v * sizeof(C));
  if (e != cudaSuccess) { release_batch(); set_cuda_error("batched solve workspace", e); return 1; }
  if (bs.ops.init(R, n, s.stream)) { release_batch(); return 1; }
  bs.R = R;
  bs.cap = R;
  bs.n = n;
  return 0;
}

// full (3*NAT) RHS r of a host or device array -> compact slot
static int to_compact(const void* src, bool dev, int r, C* dst) {
  const size_t full = (size_t)3 * s.eng.g.nat;
  const C* f = (const C*)src + (size_t)r * full;
  if (!dev) {
    cudaError_t e = cudaMemcpyAsync(s.d_xf, f, full * sizeof(C), cudaMemcpyHostToDevice, s.stream);
    if (e != cudaSuccess) { set_cuda_error("batched solve H2D", e); return 1; }
    f = s.d_xf;
  }
  v_gather<float>(f, dst + (size_t)r * bs.n, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  return check_launch("batched solve gather");
}


// ---- all-FP64 engine ----
template <typename Src> __global__ void k_to_f64(const Src* a, double2* b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    b[i] = to_d(a[i]);
}

static int ensure_f64() {
  if (f64.ready) return 0;
  const Geometry& g = s.eng.g;
  int rc = f64.eng.init_geometry(g.nx, g.ny, g.nz, g.ipbc, g.nat, g.nat0, s.h_iocc, s.prep_kind == 1);
  if (rc) { release_f64(); return 1; }
  if (s.prep_kind == 1) {
    GreenArgs<double> ga;
    ga.idipint = s.green_args.idipint; ga.gamma = s.green_args.gamma;
    ga.pyd = s.green_args.pyd; ga.pzd = s.green_args.pzd;
    for (int k = 0; k < 3; ++k) { ga.ak[k] = s.green_args.ak[k]; ga.dx[k] = s.green_args.dx[k]; }
    if (f64.eng.build_green(ga)) { release_f64(); return 1; }
  } else {
    // CPU-supplied complex-float Green: widen to complex double
    const size_t gc = g.green_count();
    std::vector<double2> h(gc);
    for (size_t i = 0; i < gc; ++i) h[i] = make_double2(s.cpu_green[i].x, s.cpu_green[i].y);
    if (f64.eng.upload_green(h.data())) { release_f64(); return 1; }
  }
  const size_t cn = (size_t)3 * g.nat0;
  cudaError_t e = cudaMalloc((void**)&f64.x, cn * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&f64.y, cn * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&f64.b, cn * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&f64.ad, cn * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&f64.ao, cn * sizeof(double2));
  if (e != cudaSuccess) { set_cuda_error("FP64 engine", e); release_f64(); return 1; }
  if (f64.ops.init(s.stream)) { release_f64(); return 1; }
  f64.eng.stream = s.stream;
  f64.ready = true;
  return 0;
}


static int ensure_b64(int R) {
  const int n = 3 * s.eng.g.nat0;
  if (b64.n == n && b64.cap >= R && b64.work) {
    if (b64.R != R) {
      b64.ops.release();
      if (b64.ops.init(R, n, s.stream)) return 1;
      b64.R = R;
    }
    return 0;
  }
  release_b64();
  const size_t v = (size_t)R * n;
  cudaError_t e = cudaMalloc((void**)&b64.b, v * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b64.x, v * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b64.adia, v * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b64.aoff, v * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b64.work, (size_t)BATCH_WORK_VECTORS * v * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b64.full, (size_t)3 * s.eng.g.nat * sizeof(double2));
  if (e != cudaSuccess) { release_b64(); set_cuda_error("FP64 batched solve workspace", e); return 1; }
  if (b64.ops.init(R, n, s.stream)) { release_b64(); return 1; }
  b64.R = R;
  b64.cap = R;
  b64.n = n;
  return 0;
}

// complex-float full RHS r (host or device) -> complex-double compact slot
static int widen_to_compact(const void* src, bool dev, int r, double2* dst) {
  const size_t full = (size_t)3 * s.eng.g.nat, cn = (size_t)3 * s.eng.g.nat0;
  const C* f = (const C*)src + (size_t)r * full;
  if (!dev) {
    cudaError_t e = cudaMemcpyAsync(s.d_xf, f, full * sizeof(C), cudaMemcpyHostToDevice, s.stream);
    if (e != cudaSuccess) { set_cuda_error("FP64 batched solve H2D", e); return 1; }
    f = s.d_xf;
  }
  v_gather<float>(f, s.d_sy, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
  const unsigned gb = (unsigned)std::min<size_t>(ceil_div(cn, 256), 148 * 16);
  k_to_f64<C><<<gb, 256, 0, s.stream>>>(s.d_sy, dst, cn);
  note_launch();
  return check_launch("FP64 batched solve widen");
}

// ---- adjoint gradient ----
// g[r][site j] = -sum_c lam_c(j) dadia_c(j) p_c(j): the derivative of s^T P
// with respect to a parameter that enters A only through CXADIA at site j
// (A^T = A, so lam = A^-1 s is the adjoint solution).  FP64 accumulation.
// grad[r][occ[q]] = -sum_c lam_r[c][q] dad_r[c][q] p_r[c][q]; the per-RHS
// strides of dad and p may be 0 (one forward solution / derivative shared by
// every adjoint source)
__global__ void k_adjoint_grad(int n, int nat0, const C* lam, const C* dad, size_t dad_rs, const C* p, size_t p_rs,
                               const int* occ, C* g, size_t g_rs) {
  const int r = blockIdx.y;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nat0; q += gridDim.x * blockDim.x) {
    double gr = 0.0, gi = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t i = (size_t)c * nat0 + q;
      const double2 l = to_d(lam[(size_t)r * n + i]), d = to_d(dad[(size_t)r * dad_rs + i]),
                    v = to_d(p[(size_t)r * p_rs + i]);
      const double tr = l.x * d.x - l.y * d.y, ti = l.x * d.y + l.y * d.x;
      gr -= tr * v.x - ti * v.y;
      gi -= tr * v.y + ti * v.x;
    }
    g[(size_t)r * g_rs + occ[q]] = make_float2((float)gr, (float)gi);
  }
}

// The prepared FP32 engine, or null before a successful prepare (read-only
// access for entry points defined in other translation units).
const Engine<float>* prepared_engine() { return s.ready ? &s.eng : nullptr; }
// The device the prepared state lives on (-1 before a successful prepare).
int prepared_device() { return s.ready ? s.device : -1; }

int make_inputs(const Engine<float>& eng, int cmdpol, int nrhs, const float* k, const float2* e0, const float* x0,
                int nmat, const float2* mref, const int16_t* icomp_host, float2* b, float2* adia, cudaStream_t st);

}  // namespace ddb

using namespace ddb;

extern "C" {

DDSCAT_CUDA_API int ddscat_cuda_release(void) {
  release_state();
  clear_error();
  return 0;
}

DDSCAT_CUDA_API const char* ddscat_cuda_last_error(void) { return last_error_text(); }

DDSCAT_CUDA_API int ddscat_cuda_prepare_green_f32(int nx, int ny, int nz, int ipbc, int nat, int nat0, int idipint,
                                                  float gamma, float pyd, float pzd, float akx, float aky, float akz,
                                                  float dx1, float dx2, float dx3, const int16_t* iocc) {
  clear_error();
  if (nx <= 0 || ny <= 0 || nz <= 0 || nat <= 0 || nat0 <= 0 || nat0 > nat || (ipbc != 0 && ipbc != 1) ||
      (idipint != 0 && idipint != 1) || !iocc || (long long)nx * ny * nz != (long long)nat) {
    set_error("prepare_green", "invalid argument");
    return 201;
  }
  if (ipbc && gamma <= 0.f) { set_error("prepare_green", "GAMMA must be >0 for PBC"); return 202; }
  release_state();
  int rc = s.eng.init_geometry(nx, ny, nz, ipbc, nat, nat0, iocc, true);
  if (rc) { release_state(); return rc == 2 ? 208 : 204; }
  GreenArgs<float> ga;
  ga.idipint = idipint; ga.gamma = gamma; ga.pyd = pyd; ga.pzd = pzd;
  ga.ak[0] = akx; ga.ak[1] = aky; ga.ak[2] = akz;
  ga.dx[0] = dx1; ga.dx[1] = dx2; ga.dx[2] = dx3;
  rc = s.eng.build_green(ga);
  if (rc) { release_state(); return 220 + rc; }
  rc = allocate_runtime();
  if (rc) { release_state(); return rc; }
  s.prep_kind = 1;
  s.green_args = ga;
  s.h_iocc = new int16_t[nat];
  std::memcpy(s.h_iocc, iocc, (size_t)nat * sizeof(int16_t));
  cudaGetDevice(&s.device);
  s.ready = true;
  return 0;
}

DDSCAT_CUDA_API int ddscat_cuda_prepare_f32(int nx, int ny, int nz, int ipbc, int nat, int nat0, const void* green,
                                            const int16_t* iocc) {
  clear_error();
  if (nx <= 0 || ny <= 0 || nz <= 0 || nat <= 0 || nat0 <= 0 || nat0 > nat || (ipbc != 0 && ipbc != 1) || !green ||
      !iocc || (long long)nx * ny * nz != (long long)nat) {
    set_error("prepare", "invalid argument");
    return 1;
  }
  release_state();
  int rc = s.eng.init_geometry(nx, ny, nz, ipbc, nat, nat0, iocc);
  if (rc) { release_state(); return rc == 2 ? 6 : 2; }
  if (allocate_runtime()) { release_state(); return 2; }
  if (s.eng.upload_green(green)) { release_state(); return 4; }
  s.prep_kind = 2;
  s.cpu_green.assign((const float2*)green, (const float2*)green + s.eng.g.green_count());
  s.h_iocc = new int16_t[nat];
  std::memcpy(s.h_iocc, iocc, (size_t)nat * sizeof(int16_t));
  cudaGetDevice(&s.device);
  s.ready = true;
  return 0;
}

DDSCAT_CUDA_API int ddscat_cuda_apply_f32(int cwhat, const void* x, void* y, const void* adia, const void* aoff) {
  if (!s.ready) { set_error("apply", "not prepared"); return 10; }
  if ((cwhat != 'N' && cwhat != 'C') || !x || !y || !adia || !aoff) { set_error("apply", "invalid argument"); return 11; }
  const size_t b = (size_t)3 * s.eng.g.nat * sizeof(C);
  cudaError_t e = copy_h2d(s.d_xf, x, b);
  if (e != cudaSuccess) { set_cuda_error("x H2D", e); return 12; }
  e = copy_h2d(s.d_adia, adia, b);
  if (e != cudaSuccess) { set_cuda_error("adia H2D", e); return 13; }
  s.aoff_zero = all_zero(aoff, b);  // zero CXAOFF: neither copied nor read
  if (!s.aoff_zero) e = copy_h2d(s.d_aoff, aoff, b);
  if (e != cudaSuccess) { set_cuda_error("aoff H2D", e); return 14; }
  MvArgs<float> a;
  a.x = s.d_xf; a.y = s.d_yf; a.io_full = 1;
  a.adia = s.d_adia; a.aoff = s.aoff_zero ? nullptr : s.d_aoff; a.a_full = 1;
  a.conj = (cwhat == 'C'); a.nrhs = 1;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  const bool timed = verbose_level() >= 1 && cudaEventCreate(&ev[0]) == cudaSuccess &&
                     cudaEventCreate(&ev[1]) == cudaSuccess;
  if (timed) cudaEventRecord(ev[0], s.stream);
  int rc = s.eng.matvec(a);
  if (!rc) rc = matvec_check(s.eng);
  if (timed) cudaEventRecord(ev[1], s.stream);
  if (!rc) {
    e = copy_d2h(y, s.d_yf, b);
    if (e != cudaSuccess) { set_cuda_error("y D2H", e); rc = 15; }
  }
  if (timed) {
    float ms = 0.f;
    if (!rc && cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) report_matvec_line(cwhat, "host-copy", ms);
  }
  if (ev[0]) cudaEventDestroy(ev[0]);
  if (ev[1]) cudaEventDestroy(ev[1]);
  cudaGetLastError();  // a failed event creation leaves no sticky error behind
  return rc;
}

#define SOLVER_ENTRY(fname, fn, nm, inv, ws, h2d, d2h, pub)                                                          \
  DDSCAT_CUDA_API int fname(const void* b, void* x, const void* adia, const void* aoff, int ndim, int maxit, float tol, \
                            int* itno, float* tole, int* ncompte) {                                                   \
    static const SolverCodes sc{nm, inv, ws, h2d, d2h, pub};                                                          \
    return run_solver(sc, fn<float>, b, x, adia, aoff, ndim, maxit, tol, itno, tole, ncompte);                        \
  }
SOLVER_ENTRY(ddscat_cuda_solve_gpbicg_f32, solve_gpbicg, "GPBICG", 30, 29, 31, 40, false)
SOLVER_ENTRY(ddscat_cuda_solve_qmrccg_f32, solve_qmrccg, "QMRCCG", 50, 29, 51, 61, false)
SOLVER_ENTRY(ddscat_cuda_solve_pbcgst_f32, solve_pbcgst, "PBCGST", 70, 29, 71, 86, true)
SOLVER_ENTRY(ddscat_cuda_solve_pbcgs2_f32, solve_pbcgs2, "PBCGS2", 90, 29, 91, 107, false)
SOLVER_ENTRY(ddscat_cuda_solve_petrkp_f32, solve_petrkp, "PETRKP", 110, 29, 111, 124, false)
SOLVER_ENTRY(ddscat_cuda_solve_bicgstab4_f32, solve_bicgstab4, "BiCGStab4", 130, 131, 131, 145, false)
SOLVER_ENTRY(ddscat_cuda_solve_gpbicgstab2_f32, solve_gpbicgstab2, "GPBiCGStab2", 150, 151, 151, 173, false)
SOLVER_ENTRY(ddscat_cuda_solve_gpbicgstab4_f32, solve_gpbicgstab4, "GPBiCGStab4", 180, 181, 181, 207, false)
#undef SOLVER_ENTRY

DDSCAT_CUDA_API int ddscat_cuda_evalq_f32(int use_resident, const void* e_compact, const void* p_compact,
                                          const void* adia_compact, const void* aoff_compact, float akx, float aky,
                                          float akz, float e02, double* cabs, double* cext, double* cpha) {
  clear_error();
  if (!s.ready || !cabs || !cext || !cpha || !(e02 > 0.f)) { set_error("GPU EVALQ", "invalid argument"); return 300; }
  const size_t cn = (size_t)3 * s.eng.g.nat0, cb = cn * sizeof(C);
  const C *ad = s.d_adia, *ao = s.aoff_zero ? nullptr : s.d_aoff;
  int a_full = 1;
  if (use_resident) {
    if (!s.solution_valid) { set_error("GPU EVALQ", "no resident final polarization published by solver"); return 301; }
  } else {
    if (!e_compact || !p_compact || !adia_compact || !aoff_compact) {
      set_error("GPU EVALQ", "missing compact host arrays");
      return 302;
    }
    cudaError_t e = cudaMemcpy(s.d_b, e_compact, cb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s.d_sx, p_compact, cb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { set_cuda_error("GPU EVALQ E/P H2D", e); return 303; }
    s.solution_valid = true;
    C* tad = s.d_work;  // compact operator copies live in the Krylov workspace
    C* tao = s.d_work + cn;
    e = cudaMemcpy(tad, adia_compact, cb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tao, aoff_compact, cb, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { set_cuda_error("GPU EVALQ ADIA/AOFF H2D", e); return 305; }
    ad = tad;
    ao = all_zero(aoff_compact, cb) ? nullptr : tao;
    a_full = 0;
  }
  const double ak2 = (double)akx * akx + (double)aky * aky + (double)akz * akz, akk = std::sqrt(ak2), ak3 = akk * ak2;
  double2 zabs, zep;
  int rc = evalq_compute<float>(s.eng, s.ops, s.d_b, s.d_sx, ad, ao, a_full, s.d_sy, ak3, &zabs, &zep);
  if (rc) return rc;
  const double pi = 4.0 * std::atan(1.0);
  *cabs = -4.0 * pi * akk * zabs.y / (double)e02;
  *cext = 4.0 * pi * akk * zep.y / (double)e02;
  *cpha = 2.0 * pi * akk * zep.x / (double)e02;
  return 0;
}

DDSCAT_CUDA_API int ddscat_cuda_scat_f32(int jpbc, int ndir, const float* ak, const float* aks, const float* dx,
                                         const float* em1, const float* em2, float e02, float etasca, const void* e01v,
                                         const float* x0, double* cbksca, double* csca, double* cscag, double* cscag2,
                                         int* navg, void* f1v, void* f2v) {
  clear_error();
  if (!s.ready || !s.solution_valid || !ak || !dx || !x0 || !cbksca || !csca || !cscag || !cscag2 || !navg ||
      !(e02 > 0.f)) {
    set_error("GPU SCAT", "invalid state/argument");
    return 320;
  }
  if (ndir > 0 && (!aks || !em1 || !em2 || !f1v || !f2v)) {
    set_error("GPU SCAT", "missing selected-direction arrays");
    return 321;
  }
  const double ak2 = (double)ak[0] * ak[0] + (double)ak[1] * ak[1] + (double)ak[2] * ak[2], akk = std::sqrt(ak2),
               ak3 = akk * ak2;
  *cbksca = 0.0; *csca = 0.0; cscag[0] = cscag[1] = cscag[2] = 0.0; *cscag2 = 0.0; *navg = 0;
  if (jpbc == 0) {
    if (!e01v || !(etasca > 0.f)) {
      set_error("GPU SCAT", "finite-target integration needs CXE01 and ETASCA>0");
      return 323;
    }
    std::vector<IntDir> idirs;
    if (make_integration_dirs(ak, (const C*)e01v, etasca, s.eng.g.nat0, idirs)) return 324;
    const int nd = (int)idirs.size();
    *navg = nd;
    std::vector<float> hd((size_t)3 * nd);
    for (int i = 0; i < nd; ++i)
      for (int k = 0; k < 3; ++k) hd[3 * i + k] = idirs[i].k[k];
    std::vector<double2> sums((size_t)3 * nd);
    int rc = farfield_sums<float>(s.eng, s.d_sx, hd.data(), nd, dx, x0, sums.data(), s.stream);
    if (rc) return rc;
    scat_integrate(idirs, sums.data(), ak2, (double)e02, cbksca, csca, cscag, cscag2);
  }
  if (ndir > 0) {
    std::vector<double2> sums((size_t)3 * ndir);
    int rc = farfield_sums<float>(s.eng, s.d_sx, aks, ndir, dx, x0, sums.data(), s.stream);
    if (rc) return rc == 325 ? 330 : rc;
    const double term = ak3 / std::sqrt((double)e02);
    C* h1 = (C*)f1v;
    C* h2 = (C*)f2v;
    for (int i = 0; i < ndir; ++i) {
      const double2 sx = sums[3 * i], sy = sums[3 * i + 1], sz = sums[3 * i + 2];
      const double a1r = em1[3 * i] * sx.x + em1[3 * i + 1] * sy.x + em1[3 * i + 2] * sz.x;
      const double a1i = em1[3 * i] * sx.y + em1[3 * i + 1] * sy.y + em1[3 * i + 2] * sz.y;
      const double a2r = em2[3 * i] * sx.x + em2[3 * i + 1] * sy.x + em2[3 * i + 2] * sz.x;
      const double a2i = em2[3 * i] * sx.y + em2[3 * i + 1] * sy.y + em2[3 * i + 2] * sz.y;
      h1[i] = make_float2((float)(term * a1r), (float)(term * a1i));
      h2[i] = make_float2((float)(term * a2r), (float)(term * a2i));
    }
  }
  return 0;
}

// Torque cross sections of the resident solution (DDSCAT's DOTORQ branch of
// SCAT, getfml_cuda.f90:1135-1144, whose torque sums the reference leaves to
// DDSCAT's CPU SCAT).  Physics restated in the oracle (scat_torque):
//   C_inc  = 8 pi k / E02 sum_j [1/2 Re(P_j x E_j*) + (1/2) Im(P_j . E_j*) r_j x k]
//   C_flux = k^4 / E02 sum_d w_d Im[-i k n x V - (n.S)(n x e*) + e* x e]
// with e = S - n (n.S), V_b = sum_a e_a* U_ab over SCAT's integration directions.
extern "C" DDSCAT_CUDA_API int ddscat_b200_scat_torque_f32(const float* ak, const float* dx, float e02, float etasca,
                                                          const void* e01v, const float* x0, double* ctrq_inc,
                                                          double* ctrq_flux, int* navg) {
  clear_error();
  if (!s.ready || !s.solution_valid || !ak || !dx || !x0 || !e01v || !ctrq_inc || !ctrq_flux || !navg ||
      !(e02 > 0.f) || !(etasca > 0.f)) {
    set_error("GPU torque", "invalid state/argument");
    return 340;
  }
  const double ak2 = (double)ak[0] * ak[0] + (double)ak[1] * ak[1] + (double)ak[2] * ak[2], akk = std::sqrt(ak2);
  const double pi = 4.0 * std::atan(1.0);
  const double kd[3] = {ak[0], ak[1], ak[2]};
  double gam[6];
  int rc = incident_torque<float>(s.eng, s.d_sx, s.d_b, dx, x0, kd, gam, s.stream);
  if (rc) return rc;
  for (int k = 0; k < 3; ++k) ctrq_inc[k] = 8.0 * pi * akk * (gam[k] + gam[3 + k]) / (double)e02;
  std::vector<IntDir> idirs;
  if (make_integration_dirs(ak, (const C*)e01v, etasca, s.eng.g.nat0, idirs)) return 344;
  const int nd = (int)idirs.size();
  *navg = nd;
  std::vector<double> hd((size_t)3 * nd);
  for (int i = 0; i < nd; ++i)
    for (int k = 0; k < 3; ++k) hd[3 * i + k] = idirs[i].k[k];
  std::vector<double2> sums((size_t)12 * nd);
  rc = farfield_torque_sums<float>(s.eng, s.d_sx, hd.data(), nd, dx, x0, sums.data(), s.stream);
  if (rc) return rc == 325 ? 345 : rc;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < nd; ++i) {
    const double2* q = &sums[(size_t)12 * i];
    double n[3];
    for (int k = 0; k < 3; ++k) n[k] = hd[3 * i + k] / akk;
    const double nsr = n[0] * q[0].x + n[1] * q[1].x + n[2] * q[2].x, nsi = n[0] * q[0].y + n[1] * q[1].y + n[2] * q[2].y;
    double er[3], ei[3];
    for (int a = 0; a < 3; ++a) { er[a] = q[a].x - n[a] * nsr; ei[a] = q[a].y - n[a] * nsi; }
    // V_b = sum_a conj(e_a) U_ab
    double vr[3], vi[3];
    for (int b = 0; b < 3; ++b) {
      vr[b] = vi[b] = 0.0;
      for (int a = 0; a < 3; ++a) {
        const double2 u = q[3 + 3 * a + b];
        vr[b] += er[a] * u.x + ei[a] * u.y;
        vi[b] += er[a] * u.y - ei[a] * u.x;
      }
    }
    for (int c = 0; c < 3; ++c) {
      const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      // Im(-i k (n x V)_c) = -k Re((n x V)_c)
      const double t1 = -akk * (n[c1] * vr[c2] - n[c2] * vr[c1]);
      // Im(-(n.S)(n x e*)_c), (n x e*)_c = n_c1 conj(e_c2) - n_c2 conj(e_c1)
      const double xr = n[c1] * er[c2] - n[c2] * er[c1], xi = -(n[c1] * ei[c2] - n[c2] * ei[c1]);
      const double t2 = -(nsr * xi + nsi * xr);
      // Im((e* x e)_c) = Im(conj(e_c1) e_c2 - conj(e_c2) e_c1) = 2 (er_c1 ei_c2 - ei_c1 er_c2)
      const double t3 = 2.0 * (er[c1] * ei[c2] - ei[c1] * er[c2]);
      acc[c] += idirs[i].w[0] * (t1 + t2 + t3);
    }
  }
  const double fac = ak2 * ak2 / (double)e02;
  for (int k = 0; k < 3; ++k) ctrq_flux[k] = fac * acc[k];
  return 0;
}

// ---- library extensions (declared in ddscat_b200.h) ----
DDSCAT_CUDA_API int ddscat_b200_set_verbose(int level) {
  g_verbose = level < 0 ? -1 : (level > 2 ? 2 : level);
  return 0;
}

DDSCAT_CUDA_API int ddscat_b200_layout(void) { return slices_build(); }

DDSCAT_CUDA_API unsigned long long ddscat_b200_launch_count(void) { return g_launches.load(); }

DDSCAT_CUDA_API int ddscat_b200_solve_batch_f32(int solver, int nrhs, const void* b, void* x, const void* adia,
                                                const void* aoff, int maxit, float tol, int* itno, float* tole,
                                                int* ncompte, int* status) {
  clear_error();
  if (!s.ready || nrhs <= 0 || !b || !x || !adia || maxit <= 0 || !(tol > 0.f) || !itno || !tole || !ncompte ||
      !status) {
    set_error("batched solve", "invalid argument or not prepared");
    return 500;
  }
  const int replace = (solver & DDSCAT_B200_REPLACE_RESIDUAL) != 0;
  const int sym = (solver & DDSCAT_B200_QMR_SYMMETRIC) != 0;
  const int graph = (solver & DDSCAT_B200_GRAPH) != 0;
  solver &= ~(DDSCAT_B200_REPLACE_RESIDUAL | DDSCAT_B200_QMR_SYMMETRIC | DDSCAT_B200_GRAPH);
  if (sym && solver != DDSCAT_B200_QMRCCG) {
    set_error("batched solve", "DDSCAT_B200_QMR_SYMMETRIC applies to QMRCCG only");
    return 501;
  }
  if (solver != DDSCAT_B200_QMRCCG && solver != DDSCAT_B200_PBCGS2) {
    set_error("batched solve", "unsupported solver (QMRCCG=1, PBCGS2=2)");
    return 501;
  }
  const bool dev = is_device_ptr(b);
  if (is_device_ptr(x) != dev || is_device_ptr(adia) != dev || (aoff && is_device_ptr(aoff) != dev)) {
    set_error("batched solve", "b, x, adia, aoff must all be host or all be device pointers");
    return 502;
  }
  if (ensure_batch(nrhs)) return 503;
  const size_t full = (size_t)3 * s.eng.g.nat;
  bool use_aoff = aoff != nullptr;
  if (use_aoff && !dev) use_aoff = !all_zero(aoff, nrhs * full * sizeof(C));
  for (int r = 0; r < nrhs; ++r) {
    if (to_compact(b, dev, r, bs.b) || to_compact(x, dev, r, bs.x) || to_compact(adia, dev, r, bs.adia)) return 504;
    if (use_aoff && to_compact(aoff, dev, r, bs.aoff)) return 504;
  }
  BatchIO<float> io;
  io.eng = &s.eng; io.ops = &bs.ops; io.R = nrhs; io.n = bs.n;
  io.b = bs.b; io.x = bs.x; io.adia = bs.adia; io.aoff = use_aoff ? bs.aoff : nullptr;
  io.work = bs.work; io.nwork = BATCH_WORK_VECTORS;
  io.maxit = maxit; io.tol = (double)tol; io.verbose = verbose_level() >= 2; io.replace = replace; io.sym = sym;
  io.graph = graph;
  BatchResult res;
  int rc = solver == DDSCAT_B200_QMRCCG ? solve_batch_qmrccg<float>(io, res) : solve_batch_pbcgs2<float>(io, res);
  if (!rc) rc = matvec_check(s.eng);
  bs.matvec_ms = io.matvec_ms;
  bs.matvec_rhs = io.matvec_rhs;
  bs.matvec_calls = io.matvec_calls;
  if (rc) return rc == 1 ? 505 : rc;
  // solutions back to the caller's full layout (zeros on vacuum sites)
  for (int r = 0; r < nrhs; ++r) {
    C* dst = dev ? (C*)x + (size_t)r * full : s.d_xf;
    cudaError_t e = cudaMemsetAsync(dst, 0, full * sizeof(C), s.stream);
    if (e != cudaSuccess) { set_cuda_error("batched solve output", e); return 506; }
    v_scatter<float>(bs.x + (size_t)r * bs.n, dst, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
    if (check_launch("batched solve scatter")) return 506;
    if (!dev) {
      e = cudaMemcpyAsync((C*)x + (size_t)r * full, s.d_xf, full * sizeof(C), cudaMemcpyDeviceToHost, s.stream);
      if (e != cudaSuccess) { set_cuda_error("batched solve D2H", e); return 506; }
    }
  }
  cudaError_t e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) { set_cuda_error("batched solve", e); return 506; }
  int worst = 0;
  for (int r = 0; r < nrhs; ++r) {
    itno[r] = res.itno[r];
    tole[r] = (float)res.tole[r];
    ncompte[r] = res.ncompte[r];
    status[r] = res.status[r];
    if (res.status[r] && !worst) worst = res.status[r];
  }
  if (worst) {
    char msg[128];
    std::snprintf(msg, sizeof(msg), "at least one right-hand side broke down (first status %d)", worst);
    set_error("batched solve", msg);
  }
  return 0;
}

DDSCAT_CUDA_API int ddscat_b200_last_solve_stats(double* matvec_ms, long long* rhs_matvecs, int* matvec_calls) {
  if (matvec_ms) *matvec_ms = bs.matvec_ms;
  if (rhs_matvecs) *rhs_matvecs = bs.matvec_rhs;
  if (matvec_calls) *matvec_calls = bs.matvec_calls;
  return 0;
}

DDSCAT_CUDA_API int ddscat_b200_residual_f64(int nrhs, const void* b, const void* x, const void* adia, const void* aoff,
                                             double* resid) {
  clear_error();
  if (!s.ready || nrhs <= 0 || !b || !x || !adia || !resid) { set_error("FP64 residual", "invalid argument"); return 510; }
  const bool dev = is_device_ptr(b);
  if (ensure_f64()) return 511;
  const size_t full = (size_t)3 * s.eng.g.nat, cn = (size_t)3 * s.eng.g.nat0;
  const unsigned gb = (unsigned)std::min<size_t>(ceil_div(cn, 256), 148 * 16);
  C* tmp = s.d_sy;  // compact float staging
  for (int r = 0; r < nrhs; ++r) {
    const void* srcs[4] = {b, x, adia, aoff};
    double2* dsts[4] = {f64.b, f64.x, f64.ad, f64.ao};
    for (int k = 0; k < 4; ++k) {
      if (!srcs[k]) continue;
      const C* f = (const C*)srcs[k] + (size_t)r * full;
      if (!dev) {
        cudaError_t e = cudaMemcpyAsync(s.d_xf, f, full * sizeof(C), cudaMemcpyHostToDevice, s.stream);
        if (e != cudaSuccess) { set_cuda_error("FP64 residual H2D", e); return 512; }
        f = s.d_xf;
      }
      v_gather<float>(f, tmp, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
      k_to_f64<C><<<gb, 256, 0, s.stream>>>(tmp, dsts[k], cn);
      note_launch();
      if (check_launch("FP64 residual widen")) return 512;
    }
    MvArgs<double> a;
    a.x = f64.x; a.y = f64.y; a.io_full = 0;
    a.adia = f64.ad; a.aoff = aoff ? f64.ao : nullptr; a.a_full = 0; a.nrhs = 1;
    int rc = f64.eng.matvec(a);
    if (rc) return rc;
    int err = 0;
    const double bn = f64.ops.nrm2((int)cn, f64.b, &err);
    const double rn = f64.ops.norm_diff((int)cn, f64.b, f64.y, &err);
    if (err) return 513;
    resid[r] = bn > 0.0 ? rn / bn : INFINITY;
  }
  return 0;
}

DDSCAT_CUDA_API int ddscat_b200_autotune_f32(int iters, float* default_ms, float* best_ms) {
  clear_error();
  if (!s.ready || iters <= 0 || !default_ms || !best_ms) {
    set_error("autotune", "invalid argument or not prepared");
    return 410;
  }
  return autotune_engine(s.eng, iters, default_ms, best_ms) ? 411 : 0;
}

DDSCAT_CUDA_API int ddscat_b200_matvec_timing(int nrhs, int iters, int cwhat, float* ms_per_call) {
  clear_error();
  if (!s.ready || nrhs <= 0 || iters <= 0 || !ms_per_call || (cwhat != 'N' && cwhat != 'C')) {
    set_error("matvec_timing", "invalid argument");
    return 400;
  }
  const size_t cn = (size_t)3 * s.eng.g.nat0;
  C *x = nullptr, *y = nullptr, *ad = nullptr;
  cudaError_t e = cudaMalloc((void**)&x, cn * nrhs * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&y, cn * nrhs * sizeof(C));
  if (e == cudaSuccess) e = cudaMalloc((void**)&ad, cn * nrhs * sizeof(C));
  if (e != cudaSuccess) { cudaFree(x); cudaFree(y); cudaFree(ad); set_cuda_error("matvec_timing", e); return 401; }
  {
    std::vector<C> h(cn);
    for (size_t i = 0; i < cn; ++i) h[i] = make_float2((float)((i * 2654435761u) % 1000) * 1e-3f, (float)(i % 7) * 0.1f);
    for (int r = 0; r < nrhs; ++r) {
      cudaMemcpy(x + r * cn, h.data(), cn * sizeof(C), cudaMemcpyHostToDevice);
      cudaMemcpy(ad + r * cn, h.data(), cn * sizeof(C), cudaMemcpyHostToDevice);
    }
  }
  MvArgs<float> a;
  a.x = x; a.x_rs = cn; a.y = y; a.y_rs = cn; a.io_full = 0;
  a.adia = ad; a.a_rs = cn; a.a_full = 0; a.aoff = nullptr; a.conj = (cwhat == 'C'); a.nrhs = nrhs;
  int rc = 0;
  for (int w = 0; w < 3 && !rc; ++w) rc = s.eng.matvec(a);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s.stream);
  for (int i = 0; i < iters && !rc; ++i) rc = s.eng.matvec(a);
  cudaEventRecord(e1, s.stream);
  e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(x); cudaFree(y); cudaFree(ad);
  if (!rc && e != cudaSuccess) { set_cuda_error("matvec_timing", e); rc = 402; }
  if (!rc) rc = matvec_check(s.eng);
  *ms_per_call = ms / iters;
  return rc;
}

}  // extern "C"

extern "C" DDSCAT_CUDA_API int ddscat_b200_mueller_f32(int ndir, const float* ak, const void* e01, const void* e02,
                                                       const float* em2, const void* f11, const void* f21,
                                                       const void* f12, const void* f22, void* s1234, double* smat) {
  clear_error();
  if (ndir <= 0 || !ak || !e01 || !e02 || !em2 || !f11 || !f21 || !f12 || !f22 || !smat) {
    set_error("Mueller", "invalid argument");
    return 700;
  }
  return mueller_compute(ndir, ak, static_cast<const float2*>(e01), static_cast<const float2*>(e02), em2,
                         static_cast<const float2*>(f11), static_cast<const float2*>(f21),
                         static_cast<const float2*>(f12), static_cast<const float2*>(f22),
                         static_cast<float2*>(s1234), smat);
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_mueller_f64(int ndir, const double* ak, const void* e01, const void* e02,
                                                       const double* em2, const void* f11, const void* f21,
                                                       const void* f12, const void* f22, void* s1234, double* smat) {
  clear_error();
  if (ndir <= 0 || !ak || !e01 || !e02 || !em2 || !f11 || !f21 || !f12 || !f22 || !smat) {
    set_error("Mueller FP64", "invalid argument");
    return 700;
  }
  return mueller_compute_f64(ndir, ak, static_cast<const double2*>(e01), static_cast<const double2*>(e02), em2,
                             static_cast<const double2*>(f11), static_cast<const double2*>(f21),
                             static_cast<const double2*>(f12), static_cast<const double2*>(f22),
                             static_cast<double2*>(s1234), smat);
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_scat_amplitudes_f64(int nrhs, const void* x, int ndir, const double* ak,
                                                               const double* aks, const double* em1,
                                                               const double* em2, const double* dx, const double* x0,
                                                               double e02, void* f1, void* f2) {
  clear_error();
  if (!s.ready || nrhs <= 0 || ndir <= 0 || !x || !ak || !aks || !em1 || !em2 || !dx || !x0 || !(e02 > 0.0) || !f1 ||
      !f2) {
    set_error("FP64 amplitudes", "invalid argument or not prepared");
    return 710;
  }
  const Geometry& g = s.eng.g;
  const size_t full = (size_t)3 * g.nat, cn = (size_t)3 * g.nat0;
  const bool dev = is_device_ptr(x);
  double2 *d_full = nullptr, *d_p = nullptr;
  cudaError_t e = cudaSuccess;
  if (!dev) e = cudaMalloc((void**)&d_full, full * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_p, cn * sizeof(double2));
  if (e != cudaSuccess) {
    cudaFree(d_full);
    set_cuda_error("FP64 amplitudes workspace", e);
    return 711;
  }
  const double kk = std::sqrt(ak[0] * ak[0] + ak[1] * ak[1] + ak[2] * ak[2]);
  const double term = kk * kk * kk / std::sqrt(e02);
  std::vector<double2> sums((size_t)3 * ndir);
  double2* h1 = static_cast<double2*>(f1);
  double2* h2 = static_cast<double2*>(f2);
  int rc = 0;
  for (int r = 0; r < nrhs && !rc; ++r) {
    const double2* src = static_cast<const double2*>(x) + (size_t)r * full;
    if (!dev) {
      e = cudaMemcpyAsync(d_full, src, full * sizeof(double2), cudaMemcpyHostToDevice, s.stream);
      if (e != cudaSuccess) { set_cuda_error("FP64 amplitudes H2D", e); rc = 711; break; }
      src = d_full;
    }
    v_gather<double>(src, d_p, s.eng.occ, g.nat, g.nat0, s.stream);
    if (check_launch("FP64 amplitudes gather")) { rc = 712; break; }
    if (farfield_sums_f64(s.eng.occ, g.nx, g.ny, g.nz, g.nat0, d_p, aks, ndir, dx, x0, sums.data(), s.stream)) {
      rc = 712;
      break;
    }
    for (int i = 0; i < ndir; ++i) {
      const double2 sx = sums[3 * i], sy = sums[3 * i + 1], sz = sums[3 * i + 2];
      const double* a = em1 + 3 * i;
      const double* b = em2 + 3 * i;
      h1[(size_t)r * ndir + i] = make_double2(term * (a[0] * sx.x + a[1] * sy.x + a[2] * sz.x),
                                              term * (a[0] * sx.y + a[1] * sy.y + a[2] * sz.y));
      h2[(size_t)r * ndir + i] = make_double2(term * (b[0] * sx.x + b[1] * sy.x + b[2] * sz.x),
                                              term * (b[0] * sx.y + b[1] * sy.y + b[2] * sz.y));
    }
  }
  cudaFree(d_full);
  cudaFree(d_p);
  return rc;
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_scat_csca_f64(int nrhs, const void* x, const float* ak, const void* e01,
                                                        float etasca, const float* dx, const float* x0, float e02,
                                                        double* cbksca, double* csca, double* cscag,
                                                        double* cscag2, int* navg) {
  clear_error();
  if (!s.ready || nrhs <= 0 || !x || !ak || !e01 || !(etasca > 0.f) || !dx || !x0 || !(e02 > 0.f) || !cbksca ||
      !csca || !cscag || !cscag2 || !navg) {
    set_error("FP64 SCAT", "invalid argument or not prepared");
    return 710;
  }
  const Geometry& g = s.eng.g;
  const size_t full = (size_t)3 * g.nat, cn = (size_t)3 * g.nat0;
  const bool dev = is_device_ptr(x);
  double2 *d_full = nullptr, *d_p = nullptr;
  cudaError_t e = cudaSuccess;
  if (!dev) e = cudaMalloc((void**)&d_full, full * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_p, cn * sizeof(double2));
  if (e != cudaSuccess) {
    cudaFree(d_full);
    set_cuda_error("FP64 SCAT workspace", e);
    return 711;
  }
  const double ak2 = (double)ak[0] * ak[0] + (double)ak[1] * ak[1] + (double)ak[2] * ak[2];
  const double dxd[3] = {dx[0], dx[1], dx[2]}, x0d[3] = {x0[0], x0[1], x0[2]};
  int rc = 0;
  for (int r = 0; r < nrhs && !rc; ++r) {
    std::vector<IntDir> idirs;
    if (make_integration_dirs(ak, static_cast<const C*>(e01) + 3 * r, etasca, g.nat0, idirs)) { rc = 710; break; }
    const int nd = (int)idirs.size();
    navg[r] = nd;
    std::vector<double> hd((size_t)3 * nd);
    for (int i = 0; i < nd; ++i)
      for (int k = 0; k < 3; ++k) hd[3 * i + k] = (double)idirs[i].k[k];
    const double2* src = static_cast<const double2*>(x) + (size_t)r * full;
    if (!dev) {
      e = cudaMemcpyAsync(d_full, src, full * sizeof(double2), cudaMemcpyHostToDevice, s.stream);
      if (e != cudaSuccess) { set_cuda_error("FP64 SCAT H2D", e); rc = 711; break; }
      src = d_full;
    }
    v_gather<double>(src, d_p, s.eng.occ, g.nat, g.nat0, s.stream);
    if (check_launch("FP64 SCAT gather")) { rc = 712; break; }
    std::vector<double2> sums((size_t)3 * nd);
    if (farfield_sums_f64(s.eng.occ, g.nx, g.ny, g.nz, g.nat0, d_p, hd.data(), nd, dxd, x0d, sums.data(),
                          s.stream)) {
      rc = 712;
      break;
    }
    scat_integrate(idirs, sums.data(), ak2, (double)e02, cbksca + r, csca + r, cscag + 3 * r, cscag2 + r);
  }
  cudaFree(d_full);
  cudaFree(d_p);
  return rc;
}

static int make_inputs_entry(int cmdpol, int nrhs, const float* k, const void* e0, const float* x0, int nmat,
                             const void* m, const int16_t* icomp, void* b, void* adia) {
  clear_error();
  if (!s.ready || nrhs <= 0 || nmat <= 0 || !k || !e0 || !x0 || !m || (!b && !adia)) {
    set_error("make_inputs", "invalid argument or not prepared");
    return 610;
  }
  const bool dev = is_device_ptr(b ? b : adia);
  if ((b && is_device_ptr(b) != dev) || (adia && is_device_ptr(adia) != dev)) {
    set_error("make_inputs", "b and adia must both be host or both be device pointers");
    return 610;
  }
  const size_t full = (size_t)3 * s.eng.g.nat;
  float2 *db = static_cast<float2*>(b), *da = static_cast<float2*>(adia);
  float2* tmp = nullptr;
  if (!dev) {
    const size_t per = (size_t)nrhs * full;
    cudaError_t e = cudaMalloc((void**)&tmp, per * sizeof(float2) * ((b ? 1 : 0) + (adia ? 1 : 0)));
    if (e != cudaSuccess) { set_cuda_error("make_inputs staging", e); return 612; }
    db = b ? tmp : nullptr;
    da = adia ? tmp + (b ? per : 0) : nullptr;
  }
  int rc = make_inputs(s.eng, cmdpol, nrhs, k, static_cast<const float2*>(e0), x0, nmat,
                       static_cast<const float2*>(m), icomp, db, da, s.stream);
  if (!rc && !dev) {
    const size_t bytes = (size_t)nrhs * full * sizeof(float2);
    cudaError_t e = cudaSuccess;
    if (b) e = cudaMemcpy(b, db, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && adia) e = cudaMemcpy(adia, da, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_cuda_error("make_inputs D2H", e); rc = 612; }
  }
  cudaFree(tmp);
  return rc;
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_make_inputs_f32(int nrhs, const float* k, const void* e0, const float* x0,
                                                           int nmat, const void* m, const int16_t* icomp, void* b,
                                                           void* adia) {
  return make_inputs_entry(DDSCAT_B200_LATTDR, nrhs, k, e0, x0, nmat, m, icomp, b, adia);
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_make_inputs_pol_f32(int cmdpol, int nrhs, const float* k, const void* e0,
                                                               const float* x0, int nmat, const void* m,
                                                               const int16_t* icomp, void* b, void* adia) {
  return make_inputs_entry(cmdpol, nrhs, k, e0, x0, nmat, m, icomp, b, adia);
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_solve_batch_f64(int solver, int nrhs, const void* b, void* x,
                                                           const void* adia, const void* aoff, int maxit, double tol,
                                                           int* itno, double* tole, int* ncompte, int* status) {
  clear_error();
  if (!s.ready || nrhs <= 0 || !b || !x || !adia || maxit <= 0 || !(tol > 0.0) || !itno || !tole || !ncompte ||
      !status) {
    set_error("FP64 batched solve", "invalid argument or not prepared");
    return 520;
  }
  const int replace = (solver & DDSCAT_B200_REPLACE_RESIDUAL) != 0;
  const int sym = (solver & DDSCAT_B200_QMR_SYMMETRIC) != 0;
  const bool in64 = (solver & DDSCAT_B200_INPUTS_F64) != 0;
  solver &= ~(DDSCAT_B200_REPLACE_RESIDUAL | DDSCAT_B200_QMR_SYMMETRIC | DDSCAT_B200_INPUTS_F64);
  if ((solver != DDSCAT_B200_QMRCCG && solver != DDSCAT_B200_PBCGS2) || (sym && solver != DDSCAT_B200_QMRCCG)) {
    set_error("FP64 batched solve", "unsupported solver or flag");
    return 521;
  }
  const bool dev = is_device_ptr(b);
  if (is_device_ptr(x) != dev || is_device_ptr(adia) != dev || (aoff && is_device_ptr(aoff) != dev)) {
    set_error("FP64 batched solve", "b, x, adia, aoff must all be host or all be device pointers");
    return 522;
  }
  if (ensure_f64() || ensure_b64(nrhs)) return 523;
  const size_t full = (size_t)3 * s.eng.g.nat;
  // complex-double full RHS r (host or device) -> compact slot
  auto gather64 = [&](const void* src, int r, double2* dst) -> int {
    const double2* f = (const double2*)src + (size_t)r * full;
    if (!dev) {
      cudaError_t e = cudaMemcpyAsync(b64.full, f, full * sizeof(double2), cudaMemcpyHostToDevice, s.stream);
      if (e != cudaSuccess) { set_cuda_error("FP64 batched solve H2D", e); return 1; }
      f = b64.full;
    }
    v_gather<double>(f, dst, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
    return check_launch("FP64 batched solve gather");
  };
  auto load = [&](const void* src, int r, double2* dst) -> int {
    return in64 ? gather64(src, r, dst) : widen_to_compact(src, dev, r, dst);
  };
  for (int r = 0; r < nrhs; ++r) {
    if (load(b, r, b64.b + (size_t)r * b64.n) || load(adia, r, b64.adia + (size_t)r * b64.n) ||
        (aoff && load(aoff, r, b64.aoff + (size_t)r * b64.n)))
      return 524;
    const double2* xf = (const double2*)x + (size_t)r * full;
    if (!dev) {
      cudaError_t e = cudaMemcpyAsync(b64.full, xf, full * sizeof(double2), cudaMemcpyHostToDevice, s.stream);
      if (e != cudaSuccess) { set_cuda_error("FP64 batched solve H2D", e); return 524; }
      xf = b64.full;
    }
    v_gather<double>(xf, b64.x + (size_t)r * b64.n, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
    if (check_launch("FP64 batched solve gather")) return 524;
  }
  BatchIO<double> io;
  io.eng = &f64.eng; io.ops = &b64.ops; io.R = nrhs; io.n = b64.n;
  io.b = b64.b; io.x = b64.x; io.adia = b64.adia; io.aoff = aoff ? b64.aoff : nullptr;
  io.work = b64.work; io.nwork = BATCH_WORK_VECTORS;
  io.maxit = maxit; io.tol = tol; io.verbose = verbose_level() >= 2; io.replace = replace; io.sym = sym;
  BatchResult res;
  const int rc = solver == DDSCAT_B200_QMRCCG ? solve_batch_qmrccg<double>(io, res) : solve_batch_pbcgs2<double>(io, res);
  if (rc) return rc == 1 ? 525 : rc;
  for (int r = 0; r < nrhs; ++r) {
    double2* dst = dev ? (double2*)x + (size_t)r * full : b64.full;
    cudaError_t e = cudaMemsetAsync(dst, 0, full * sizeof(double2), s.stream);
    if (e != cudaSuccess) { set_cuda_error("FP64 batched solve output", e); return 526; }
    v_scatter<double>(b64.x + (size_t)r * b64.n, dst, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
    if (check_launch("FP64 batched solve scatter")) return 526;
    if (!dev) {
      e = cudaMemcpyAsync((double2*)x + (size_t)r * full, b64.full, full * sizeof(double2), cudaMemcpyDeviceToHost,
                          s.stream);
      if (e != cudaSuccess) { set_cuda_error("FP64 batched solve D2H", e); return 526; }
    }
  }
  cudaError_t e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) { set_cuda_error("FP64 batched solve", e); return 526; }
  int worst = 0;
  for (int r = 0; r < nrhs; ++r) {
    itno[r] = res.itno[r];
    tole[r] = res.tole[r];
    ncompte[r] = res.ncompte[r];
    status[r] = res.status[r];
    if (res.status[r] && !worst) worst = res.status[r];
  }
  if (worst) {
    set_error("FP64 batched solve", "at least one right-hand side stopped on a breakdown (see status)");
    return worst;
  }
  return 0;
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_adjoint_f32(int nrhs, const void* p, const void* src, const void* adia,
                                                       const void* dadia, int maxit, float tol, void* grad, void* lam,
                                                       int* itno, float* tole) {
  clear_error();
  if (!s.ready || nrhs <= 0 || !p || !src || !adia || !dadia || !grad || maxit <= 0 || !(tol > 0.f) || !itno ||
      !tole) {
    set_error("adjoint", "invalid argument or not prepared");
    return 530;
  }
  const bool dev = is_device_ptr(p);
  if (is_device_ptr(src) != dev || is_device_ptr(adia) != dev || is_device_ptr(dadia) != dev ||
      is_device_ptr(grad) != dev || (lam && is_device_ptr(lam) != dev)) {
    set_error("adjoint", "all arrays must be host or all device pointers");
    return 531;
  }
  if (ensure_batch(nrhs)) return 532;
  const size_t full = (size_t)3 * s.eng.g.nat, nat = (size_t)s.eng.g.nat;
  C* pc = bs.work + (size_t)(BATCH_WORK_VECTORS - 2) * nrhs * bs.n;  // outside the solver's slots
  C* dc = bs.aoff;
  for (int r = 0; r < nrhs; ++r) {
    if (to_compact(src, dev, r, bs.b) || to_compact(adia, dev, r, bs.adia)) return 533;
  }
  cudaError_t e = cudaMemsetAsync(bs.x, 0, (size_t)nrhs * bs.n * sizeof(C), s.stream);
  if (e != cudaSuccess) { set_cuda_error("adjoint", e); return 533; }
  // adjoint solve A lam = s: one-MATVEC QMRCCG with residual replacement
  BatchIO<float> io;
  io.eng = &s.eng; io.ops = &bs.ops; io.R = nrhs; io.n = bs.n;
  io.b = bs.b; io.x = bs.x; io.adia = bs.adia; io.aoff = nullptr;
  io.work = bs.work; io.nwork = BATCH_WORK_VECTORS - 2;
  io.maxit = maxit; io.tol = (double)tol; io.verbose = verbose_level() >= 2; io.replace = 1; io.sym = 1;
  BatchResult res;
  int rc = solve_batch_qmrccg<float>(io, res);
  if (!rc) rc = matvec_check(s.eng);
  if (rc) return rc == 1 ? 534 : rc;
  for (int r = 0; r < nrhs; ++r) {
    itno[r] = res.itno[r];
    tole[r] = (float)res.tole[r];
    if (res.status[r]) {
      set_error("adjoint", "adjoint solve broke down for at least one right-hand side");
      return res.status[r];
    }
  }
  // forward solutions and dCXADIA/dparameter, compact
  for (int r = 0; r < nrhs; ++r) {
    const C* pf = (const C*)p + (size_t)r * full;
    const C* df = (const C*)dadia + (size_t)r * full;
    for (int k = 0; k < 2; ++k) {
      const C* f = k == 0 ? pf : df;
      if (!dev) {
        e = cudaMemcpyAsync(s.d_xf, f, full * sizeof(C), cudaMemcpyHostToDevice, s.stream);
        if (e != cudaSuccess) { set_cuda_error("adjoint H2D", e); return 533; }
        f = s.d_xf;
      }
      v_gather<float>(f, (k == 0 ? pc : dc) + (size_t)r * bs.n, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
      if (check_launch("adjoint gather")) return 533;
    }
  }
  // gradient per site (zero on vacuum)
  C* gd = dev ? static_cast<C*>(grad) : s.d_xf;  // host: stage nat sites per RHS in the full-vector buffer
  const unsigned gx = (unsigned)std::min<size_t>(ceil_div((size_t)s.eng.g.nat0, 256), 1184);
  for (int r0 = 0; r0 < nrhs; r0 += dev ? nrhs : 3) {
    const int nr = dev ? nrhs : std::min(3, nrhs - r0);  // the host staging buffer holds 3 x NAT
    e = cudaMemsetAsync(gd + (dev ? 0 : 0), 0, (size_t)nr * nat * sizeof(C), s.stream);
    if (e != cudaSuccess) { set_cuda_error("adjoint", e); return 535; }
    k_adjoint_grad<<<dim3(gx, (unsigned)nr), 256, 0, s.stream>>>(bs.n, s.eng.g.nat0, bs.x + (size_t)r0 * bs.n,
                                                                 dc + (size_t)r0 * bs.n, bs.n, pc + (size_t)r0 * bs.n,
                                                                 bs.n, s.eng.occ, gd, nat);
    note_launch();
    if (check_launch("adjoint gradient")) return 535;
    if (!dev) {
      e = cudaMemcpyAsync((C*)grad + (size_t)r0 * nat, gd, (size_t)nr * nat * sizeof(C), cudaMemcpyDeviceToHost,
                          s.stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s.stream);
      if (e != cudaSuccess) { set_cuda_error("adjoint D2H", e); return 535; }
    }
  }
  if (lam) {
    for (int r = 0; r < nrhs; ++r) {
      C* dst = dev ? (C*)lam + (size_t)r * full : s.d_xf;
      e = cudaMemsetAsync(dst, 0, full * sizeof(C), s.stream);
      if (e != cudaSuccess) { set_cuda_error("adjoint", e); return 535; }
      v_scatter<float>(bs.x + (size_t)r * bs.n, dst, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
      if (check_launch("adjoint scatter")) return 535;
      if (!dev) {
        e = cudaMemcpyAsync((C*)lam + (size_t)r * full, s.d_xf, full * sizeof(C), cudaMemcpyDeviceToHost, s.stream);
        if (e != cudaSuccess) { set_cuda_error("adjoint D2H", e); return 535; }
      }
    }
  }
  e = cudaStreamSynchronize(s.stream);
  if (e != cudaSuccess) { set_cuda_error("adjoint", e); return 535; }
  return 0;
}

// ---- adjoint gradient with the forward field recomputed (library extension) ----
extern "C" DDSCAT_CUDA_API int ddscat_b200_adjoint_fwd_f32(int nsrc, const void* e, const void* src,
                                                           const void* adia, const void* dadia, int maxit, float tol,
                                                           void* grad, void* p, int* itno, float* tole) {
  clear_error();
  if (!s.ready || nsrc <= 0 || !e || !src || !adia || !dadia || !grad || maxit <= 0 || !(tol > 0.f) || !itno ||
      !tole) {
    set_error("adjoint (forward recomputed)", "invalid argument or not prepared");
    return 530;
  }
  const bool dev = is_device_ptr(e);
  if (is_device_ptr(src) != dev || is_device_ptr(adia) != dev || is_device_ptr(dadia) != dev ||
      is_device_ptr(grad) != dev || (p && is_device_ptr(p) != dev)) {
    set_error("adjoint (forward recomputed)", "all arrays must be host or all device pointers");
    return 531;
  }
  const int R = nsrc + 1;  // slot 0: the forward system A P = E; slots 1..nsrc: A lam_k = s_k
  if (ensure_batch(R)) return 532;
  const size_t full = (size_t)3 * s.eng.g.nat, nat = (size_t)s.eng.g.nat;
  C* dc = bs.aoff;  // compact dCXADIA (one vector, shared by every source)
  if (to_compact(e, dev, 0, bs.b) || to_compact(adia, dev, 0, bs.adia) || to_compact(dadia, dev, 0, dc)) return 533;
  for (int k = 0; k < nsrc; ++k)
    if (to_compact(src, dev, k, bs.b + bs.n)) return 533;
  cudaError_t ce = cudaSuccess;
  for (int r = 1; r < R && ce == cudaSuccess; ++r)
    ce = cudaMemcpyAsync(bs.adia + (size_t)r * bs.n, bs.adia, (size_t)bs.n * sizeof(C), cudaMemcpyDeviceToDevice,
                         s.stream);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(bs.x, 0, (size_t)R * bs.n * sizeof(C), s.stream);
  if (ce != cudaSuccess) { set_cuda_error("adjoint (forward recomputed)", ce); return 533; }
  // the forward and the adjoint systems share the operator: one batched
  // one-MATVEC QMRCCG solve with residual replacement over all of them
  BatchIO<float> io;
  io.eng = &s.eng; io.ops = &bs.ops; io.R = R; io.n = bs.n;
  io.b = bs.b; io.x = bs.x; io.adia = bs.adia; io.aoff = nullptr;
  io.work = bs.work; io.nwork = BATCH_WORK_VECTORS;
  io.maxit = maxit; io.tol = (double)tol; io.verbose = verbose_level() >= 2; io.replace = 1; io.sym = 1;
  BatchResult res;
  int rc = solve_batch_qmrccg<float>(io, res);
  if (!rc) rc = matvec_check(s.eng);
  if (rc) return rc == 1 ? 534 : rc;
  for (int r = 0; r < R; ++r) {
    itno[r] = res.itno[r];
    tole[r] = (float)res.tole[r];
    if (res.status[r]) {
      set_error("adjoint (forward recomputed)", "a forward or adjoint solve broke down");
      return res.status[r];
    }
  }
  // gradient per site and source (zero on vacuum)
  C* gd = dev ? static_cast<C*>(grad) : s.d_xf;  // host: stage up to 3 sources in the full-vector buffer
  const unsigned gx = (unsigned)std::min<size_t>(ceil_div((size_t)s.eng.g.nat0, 256), 1184);
  for (int k0 = 0; k0 < nsrc; k0 += dev ? nsrc : 3) {
    const int nk = dev ? nsrc : std::min(3, nsrc - k0);
    ce = cudaMemsetAsync(gd, 0, (size_t)nk * nat * sizeof(C), s.stream);
    if (ce != cudaSuccess) { set_cuda_error("adjoint (forward recomputed)", ce); return 535; }
    k_adjoint_grad<<<dim3(gx, (unsigned)nk), 256, 0, s.stream>>>(bs.n, s.eng.g.nat0, bs.x + (size_t)(1 + k0) * bs.n,
                                                                 dc, 0, bs.x, 0, s.eng.occ, gd, nat);
    note_launch();
    if (check_launch("adjoint gradient")) return 535;
    if (!dev) {
      ce = cudaMemcpyAsync((C*)grad + (size_t)k0 * nat, gd, (size_t)nk * nat * sizeof(C), cudaMemcpyDeviceToHost,
                           s.stream);
      if (ce == cudaSuccess) ce = cudaStreamSynchronize(s.stream);
      if (ce != cudaSuccess) { set_cuda_error("adjoint D2H", ce); return 535; }
    }
  }
  if (p) {  // the forward solution, full layout
    C* dst = dev ? static_cast<C*>(p) : s.d_xf;
    ce = cudaMemsetAsync(dst, 0, full * sizeof(C), s.stream);
    if (ce != cudaSuccess) { set_cuda_error("adjoint (forward recomputed)", ce); return 535; }
    v_scatter<float>(bs.x, dst, s.eng.occ, s.eng.g.nat, s.eng.g.nat0, s.stream);
    if (check_launch("adjoint scatter")) return 535;
    if (!dev) {
      ce = cudaMemcpyAsync(p, s.d_xf, full * sizeof(C), cudaMemcpyDeviceToHost, s.stream);
      if (ce != cudaSuccess) { set_cuda_error("adjoint D2H", ce); return 535; }
    }
  }
  ce = cudaStreamSynchronize(s.stream);
  if (ce != cudaSuccess) { set_cuda_error("adjoint (forward recomputed)", ce); return 535; }
  return 0;
}

// far-field weights: w_k[c][j] = |aks_k|^3 / sqrt(E02) em_k[c] exp(-i aks_k . r_j) on occupied sites
__global__ void k_ffweights(int nw, int nx, int ny, int nat, const double* aks, const double* em, double x00,
                            double x01, double x02, double term_scale, const int16_t* iocc, C* out) {
  const int k = blockIdx.y;
  const double kx = aks[3 * k], ky = aks[3 * k + 1], kz = aks[3 * k + 2];
  const double kk = sqrt(kx * kx + ky * ky + kz * kz), term = kk * kk * kk * term_scale;
  const double e0 = em[3 * k] * term, e1 = em[3 * k + 1] * term, e2 = em[3 * k + 2] * term;
  C* w = out + (size_t)k * 3 * nat;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nat; j += gridDim.x * blockDim.x) {
    C a = make_float2(0.f, 0.f), b = a, c = a;
    if (iocc[j]) {
      const int ix = j % nx, iy = (j / nx) % ny, iz = j / (nx * ny);
      const double ph = -(kx * (ix + 1 + x00) + ky * (iy + 1 + x01) + kz * (iz + 1 + x02));
      double sn, cs;
      sincos(ph, &sn, &cs);
      a = make_float2((float)(e0 * cs), (float)(e0 * sn));
      b = make_float2((float)(e1 * cs), (float)(e1 * sn));
      c = make_float2((float)(e2 * cs), (float)(e2 * sn));
    }
    w[j] = a;
    w[(size_t)nat + j] = b;
    w[2 * (size_t)nat + j] = c;
  }
}

extern "C" DDSCAT_CUDA_API int ddscat_b200_ffweights_f32(int nw, const double* aks, const double* em,
                                                         const double* x0, double e02, void* w) {
  clear_error();
  if (!s.ready || nw <= 0 || !aks || !em || !x0 || !(e02 > 0.0) || !w) {
    set_error("far-field weights", "invalid argument or not prepared");
    return 720;
  }
  const Geometry& g = s.eng.g;
  const bool dev = is_device_ptr(w);
  const size_t full = (size_t)3 * g.nat;
  double* d_par = nullptr;
  C* d_w = dev ? static_cast<C*>(w) : nullptr;
  cudaError_t ce = cudaMalloc((void**)&d_par, (size_t)6 * nw * sizeof(double));
  if (ce == cudaSuccess && !dev) ce = cudaMalloc((void**)&d_w, (size_t)nw * full * sizeof(C));
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_par, aks, (size_t)3 * nw * sizeof(double), cudaMemcpyHostToDevice,
                                              s.stream);
  if (ce == cudaSuccess) ce = cudaMemcpyAsync(d_par + 3 * (size_t)nw, em, (size_t)3 * nw * sizeof(double),
                                              cudaMemcpyHostToDevice, s.stream);
  int rc = 0;
  if (ce != cudaSuccess) {
    set_cuda_error("far-field weights", ce);
    rc = 721;
  } else {
    const unsigned gx = (unsigned)std::min<size_t>(ceil_div((size_t)g.nat, 256), std::max(1, 2368 / nw));
    k_ffweights<<<dim3(gx, (unsigned)nw), 256, 0, s.stream>>>(nw, g.nx, g.ny, g.nat, d_par, d_par + 3 * (size_t)nw,
                                                              x0[0], x0[1], x0[2], 1.0 / std::sqrt(e02),
                                                              s.eng.iocc, d_w);
    note_launch();
    if (check_launch("far-field weights")) rc = 722;
    if (!rc && !dev) {
      ce = cudaMemcpyAsync(w, d_w, (size_t)nw * full * sizeof(C), cudaMemcpyDeviceToHost, s.stream);
      if (ce != cudaSuccess) { set_cuda_error("far-field weights D2H", ce); rc = 721; }
    }
    if (!rc && (ce = cudaStreamSynchronize(s.stream)) != cudaSuccess) { set_cuda_error("far-field weights", ce); rc = 722; }
  }
  cudaFree(d_par);
  if (!dev) cudaFree(d_w);
  return rc;
}
