// Many targets of uneven grid size solved together (library extension; no
// counterpart in the reference, whose global state holds one target).
//
// Every target gets its own engine (geometry, Green tensor, FFT plans, MATVEC
// workspace), its own batched-solver state and its own CUDA stream.  The Green
// tensors are built first, one target after another.  With the device-driven
// PBCGS2 (DDSCAT_B200_GRAPH) every target's solve runs its first, host-driven
// iteration on a host thread of its own and then hands its iteration over to a
// coordinator: one CUDA graph holds the iterations of all targets as
// independent branches and is launched once per Krylov step until no RHS of
// any target is active, so the GPU runs the kernels of all targets side by
// side and the host does one launch per step.  Otherwise a pool of host
// threads drives the targets' batched Krylov solves, each thread taking the
// largest target not yet started; a solve synchronises only its own stream, so
// while one target waits for its inner products the kernels of the others keep
// the GPU busy.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>
#include "batch.h"
#include "ddscat_b200.h"

namespace ddb {

namespace {

struct Target {
  Engine<float> eng;
  BatchOps<float> ops;
  cudaStream_t st = nullptr;
  int R = 0, n = 0, first = 0;  // RHS count, compact length, index of the first RHS
  int nat = 0;                  // lattice sites of the caller's grid (its full-vector layout)
  int* occ = nullptr;           // compact index -> site of the caller's grid
  float2 *b = nullptr, *x = nullptr, *adia = nullptr, *work = nullptr, *full = nullptr;
  void release() {
    ops.release();
    eng.release();
    cudaFree(b); cudaFree(x); cudaFree(adia); cudaFree(work); cudaFree(full); cudaFree(occ);
    if (st) cudaStreamDestroy(st);
    *this = Target{};
  }
};

}  // namespace

int multi_solve(int nt, const int* dims, const int16_t* const* iocc, const float* ak, const int* nrhs,
                const void* const* b, void* const* x, const void* const* adia, int solver, int replace, int sym,
                int autotune, int graph, int maxit, float tol, int nthreads, int* itno, float* tole, int* ncompte,
                int* status) {
  const bool verbose = verbose_level() >= 2;
  auto now = []() { return std::chrono::steady_clock::now(); };
  const auto t0 = now();
  std::vector<Target> T(nt);
  auto cleanup = [&]() {
    for (auto& t : T) t.release();
  };
  int first = 0;
  double ph[4] = {0, 0, 0, 0};  // verbose: geometry, Green, workspace, inputs (s)
  auto lap = [&](int k, std::chrono::steady_clock::time_point& a) {
    if (!verbose) return;
    cudaDeviceSynchronize();
    const auto b = now();
    ph[k] += std::chrono::duration<double>(b - a).count();
    a = b;
  };
  for (int i = 0; i < nt; ++i) {
    Target& t = T[i];
    auto ta = now();
    const int nx = dims[3 * i], ny = dims[3 * i + 1], nz = dims[3 * i + 2];
    const int nat = nx * ny * nz;
    int nat0 = 0;
    for (int j = 0; j < nat; ++j) nat0 += iocc[i][j] != 0;
    if (nat0 == 0) { set_error("multi-target solve", "a target has no occupied site"); cleanup(); return 540; }
    if (cudaStreamCreate(&t.st) != cudaSuccess) { set_error("multi-target solve", "stream"); cleanup(); return 542; }
    // The engine's grid: each odd side extended by one vacuum plane, so that
    // every axis runs on the register-FFT pipeline (padded lengths need even
    // sides).  The occupied sites, their order (z, then y, then x) and so the
    // compact vectors are those of the caller's grid; the Green tensor depends
    // on the lags only, so the operator on them is unchanged.
    const int ex = nx + (nx & 1), ey = ny + (ny & 1), ez = nz + (nz & 1);
    const int enat = ex * ey * ez;
    std::vector<int16_t> eocc((size_t)enat, 0);
    std::vector<int> occ_h;
    occ_h.reserve(nat0);
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
          const int j = x + nx * (y + ny * z);
          if (iocc[i][j] == 0) continue;
          eocc[(size_t)x + ex * ((size_t)y + ey * z)] = iocc[i][j];
          occ_h.push_back(j);
        }
    t.nat = nat;
    if (cudaMalloc((void**)&t.occ, (size_t)nat0 * sizeof(int)) != cudaSuccess ||
        cudaMemcpy(t.occ, occ_h.data(), (size_t)nat0 * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) {
      set_error("multi-target solve", "index map");
      cleanup();
      return 542;
    }
    int rc = t.eng.init_geometry(ex, ey, ez, 0, enat, nat0, eocc.data(), true);
    if (rc) { cleanup(); return 543; }
    lap(0, ta);
    GreenArgs<float> ga;
    for (int k = 0; k < 3; ++k) ga.ak[k] = ak[3 * i + k];
    rc = t.eng.build_green(ga);
    if (rc) { cleanup(); return 543; }
    lap(1, ta);
    if (autotune) {
      float d = 0.f, bst = 0.f;
      if (autotune_engine(t.eng, 3, &d, &bst)) { cleanup(); return 543; }
    }
    t.eng.stream = t.st;
    t.R = nrhs[i];
    t.n = 3 * nat0;
    t.first = first;
    first += t.R;
    const size_t v = (size_t)t.R * t.n, full = (size_t)3 * nat;
    cudaError_t e = cudaMalloc((void**)&t.b, v * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t.x, v * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t.adia, v * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t.work, (size_t)BATCH_WORK_VECTORS * v * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc((void**)&t.full, full * sizeof(float2));
    if (e != cudaSuccess) { set_cuda_error("multi-target workspace", e); cleanup(); return 542; }
    if (t.ops.init(t.R, t.n, t.st)) { cleanup(); return 542; }
    lap(2, ta);
    // inputs: full host vectors -> compact device slots
    const void* src[3] = {b[i], x[i], adia[i]};
    float2* dst[3] = {t.b, t.x, t.adia};
    for (int r = 0; r < t.R; ++r)
      for (int k = 0; k < 3; ++k) {
        e = cudaMemcpyAsync(t.full, (const float2*)src[k] + (size_t)r * full, full * sizeof(float2),
                            cudaMemcpyHostToDevice, t.st);
        if (e != cudaSuccess) { set_cuda_error("multi-target H2D", e); cleanup(); return 544; }
        v_gather<float>(t.full, dst[k] + (size_t)r * t.n, t.occ, nat, nat0, t.st);
        if (check_launch("multi-target gather")) { cleanup(); return 544; }
      }
    lap(3, ta);
  }
  cudaDeviceSynchronize();
  const auto t1 = now();
  // largest target first
  std::vector<int> order(nt);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return T[a].eng.g.nat > T[c].eng.g.nat; });
  std::atomic<int> next{0};
  std::mutex mu;
  int first_rc = 0;
  std::string first_msg;
  // one graph for all targets: PBCGS2 with device-driven iterations (replacement)
  const bool grouped = graph && replace && solver == DDSCAT_B200_PBCGS2;
  void* group = grouped ? pg_group_create(nt) : nullptr;
  auto worker = [&](int fixed) {
    for (;;) {
      const int k = fixed >= 0 ? fixed : next++;
      if (k >= nt) return;
      Target& t = T[order[k]];
      BatchIO<float> io;
      io.eng = &t.eng; io.ops = &t.ops; io.R = t.R; io.n = t.n;
      io.b = t.b; io.x = t.x; io.adia = t.adia; io.aoff = nullptr;
      io.work = t.work; io.nwork = BATCH_WORK_VECTORS;
      io.maxit = maxit; io.tol = (double)tol; io.replace = replace; io.sym = sym; io.graph = graph;
      io.group = group;
      BatchResult res;
      int rc = solver == DDSCAT_B200_QMRCCG ? solve_batch_qmrccg<float>(io, res) : solve_batch_pbcgs2<float>(io, res);
      if (group && !io.group_joined) pg_group_leave(group);  // solved (or failed) without handing over
      const int i = order[k];
      const size_t full = (size_t)3 * t.nat;
      for (int r = 0; !rc && r < t.R; ++r) {
        cudaError_t e = cudaMemsetAsync(t.full, 0, full * sizeof(float2), t.st);
        if (e == cudaSuccess) {
          v_scatter<float>(t.x + (size_t)r * t.n, t.full, t.occ, t.nat, t.eng.g.nat0, t.st);
          e = cudaMemcpyAsync((float2*)x[i] + (size_t)r * full, t.full, full * sizeof(float2), cudaMemcpyDeviceToHost,
                              t.st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(t.st);
        if (e != cudaSuccess) { set_cuda_error("multi-target output", e); rc = 546; }
      }
      if (!rc) rc = matvec_check(t.eng);  // status word of the target's MATVEC kernels
      if (!rc) {
        for (int r = 0; r < t.R; ++r) {
          itno[t.first + r] = res.itno[r];
          tole[t.first + r] = (float)res.tole[r];
          ncompte[t.first + r] = res.ncompte[r];
          status[t.first + r] = res.status[r];
        }
      } else {
        std::lock_guard<std::mutex> lock(mu);
        if (!first_rc) { first_rc = rc == 1 ? 545 : rc; first_msg = last_error_text(); }
      }
      if (fixed >= 0) return;
    }
  };
  const int nw = grouped ? nt : std::max(1, std::min(nthreads, nt));
  std::vector<std::thread> pool;
  if (grouped) {
    // a thread per target up to the hand-over; this thread coordinates
    for (int k = 0; k < nt; ++k) pool.emplace_back(worker, k);
    const int grc = pg_group_run(group);
    for (auto& th : pool) th.join();
    pg_group_destroy(group);
    if (grc && !first_rc) { first_rc = 545; first_msg = last_error_text(); }
  } else {
    for (int w = 1; w < nw; ++w) pool.emplace_back(worker, -1);
    worker(-1);
    for (auto& th : pool) th.join();
  }
  const auto t2 = now();
  cleanup();
  if (verbose)
    std::printf("multi-target solve: %d targets, setup %.3f s (geometry %.3f, Green %.3f, workspace %.3f, inputs "
                "%.3f), solves %.3f s on %d threads\n",
                nt, std::chrono::duration<double>(t1 - t0).count(), ph[0], ph[1], ph[2], ph[3],
                std::chrono::duration<double>(t2 - t1).count(), nw);
  if (first_rc) {
    set_error("multi-target solve", first_msg.c_str());
    return first_rc;
  }
  for (int r = 0; r < first; ++r)
    if (status[r]) {
      set_error("multi-target solve", "at least one right-hand side stopped on a breakdown (see status)");
      return status[r];
    }
  return 0;
}

}  // namespace ddb

using namespace ddb;

extern "C" DDSCAT_CUDA_API int ddscat_b200_multi_solve_f32(int ntarget, const int* dims, const int16_t* const* iocc,
                                                           const float* ak, const int* nrhs, const void* const* b,
                                                           void* const* x, const void* const* adia, int solver,
                                                           int maxit, float tol, int nthreads, int* itno, float* tole,
                                                           int* ncompte, int* status) {
  clear_error();
  if (ntarget <= 0 || !dims || !iocc || !ak || !nrhs || !b || !x || !adia || maxit <= 0 || !(tol > 0.f) || !itno ||
      !tole || !ncompte || !status) {
    set_error("multi-target solve", "invalid argument");
    return 540;
  }
  for (int i = 0; i < ntarget; ++i)
    if (dims[3 * i] <= 0 || dims[3 * i + 1] <= 0 || dims[3 * i + 2] <= 0 || nrhs[i] <= 0 || !iocc[i] || !b[i] ||
        !x[i] || !adia[i]) {
      set_error("multi-target solve", "invalid target description");
      return 540;
    }
  const int replace = (solver & DDSCAT_B200_REPLACE_RESIDUAL) != 0;
  const int sym = (solver & DDSCAT_B200_QMR_SYMMETRIC) != 0;
  const int tune = (solver & DDSCAT_B200_AUTOTUNE) != 0;
  const int graph = (solver & DDSCAT_B200_GRAPH) != 0;
  solver &= ~(DDSCAT_B200_REPLACE_RESIDUAL | DDSCAT_B200_QMR_SYMMETRIC | DDSCAT_B200_AUTOTUNE | DDSCAT_B200_GRAPH);
  if ((solver != DDSCAT_B200_QMRCCG && solver != DDSCAT_B200_PBCGS2) || (sym && solver != DDSCAT_B200_QMRCCG)) {
    set_error("multi-target solve", "unsupported solver or flag");
    return 541;
  }
  if (nthreads <= 0) nthreads = std::min(ntarget, 8);
  return multi_solve(ntarget, dims, iocc, ak, nrhs, b, x, adia, solver, replace, sym, tune, graph, maxit, tol,
                     nthreads, itno, tole, ncompte, status);
}
