// Internal interfaces of the B200 DDA library (not part of the C ABI).
//
// Data layout in HBM
//   polarisation / field vectors: full  v[m*NAT + j]   (the ABI layout)
//                                 compact v[m*NAT0 + q], q = rank of occupied site j
//   zhat  : z-spectrum, [rhs][comp][kz < Mz][iy < ny][ix < nx]
//   slab  : xy spectrum of a batch of kz planes, [rhs][comp][kz][iy < ny][kx < Mx]
//   green : point-interleaved [point][6], points = octant (nz+1)(ny+1)(nx+1) (IPBC=0)
//           or the full Mz*My*Mx grid (IPBC=1); 6 = (xx,xy,xz,yy,yz,zz)
// The MATVEC is a z-first pipeline: z-forward (pad-skip, compact scatter fused)
// -> per kz batch { x-forward, y-forward * Green * y-inverse, x-inverse } ->
// z-inverse with the diagonal / off-diagonal CXZC terms and compact gather fused.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>
#include "common.cuh"
#include "fft.cuh"

namespace ddb {

// ---------------------------------------------------------------- errors
void set_error(const char* where, const char* what);
void set_cuda_error(const char* where, cudaError_t e);
const char* last_error_text();
void clear_error();
int check_launch(const char* where);
// console output level of the library (0 silent, 1 reference-style lines, 2 diagnostics)
int verbose_level();
void raise_smem_limit(const void* f);  // thread-safe, once per kernel
// an on/off environment switch: on when set to a non-empty value other than "0"
bool env_flag(const char* name);
unsigned long long launch_total();     // kernels launched so far (note_launch counter)
// count of kernels this library launched (reported by ddscat_b200_launch_count)
void note_launch(unsigned long long k = 1);

// ---------------------------------------------------------------- geometry
// M_a is the padded FFT length of axis a: 2 n_a as in the reference, or, for
// a library-built Green tensor with IPBC = 0, the next length >= 2 n_a that the
// register-FFT pipeline runs (the circulant embedding of the lags -(n-1)..n-1
// is exact for any M >= 2n - 1; the spectrum is still even per axis, so the
// octant k_a = 0..M_a/2 holds it).
struct Geometry {
  int nx = 0, ny = 0, nz = 0, Mx = 0, My = 0, Mz = 0;
  int nat = 0, nat0 = 0, ipbc = 0;
  size_t ngrid() const { return (size_t)Mx * My * Mz; }
  size_t octant() const { return (size_t)(Mx / 2 + 1) * (My / 2 + 1) * (Mz / 2 + 1); }
  bool padded() const { return Mx != 2 * nx || My != 2 * ny || Mz != 2 * nz; }
  size_t green_count() const { return ipbc == 0 ? 6 * octant() : 6 * ngrid(); }
};

// Arguments of one MATVEC launch sequence over `nrhs` right-hand sides.
template <typename T> struct MvArgs {
  const cplx<T>* x = nullptr;  // input, RHS r at x + r*x_rs
  size_t x_rs = 0;
  cplx<T>* y = nullptr;        // output, RHS r at y + r*y_rs
  size_t y_rs = 0;
  int io_full = 0;             // 1: x,y are full 3*NAT vectors; 0: compact 3*NAT0
  const cplx<T>* adia = nullptr;
  const cplx<T>* aoff = nullptr;  // null => no off-diagonal site block
  size_t a_rs = 0;                // per-RHS stride of adia/aoff (0 = shared)
  int a_full = 1;                 // adia/aoff layout: 1 full, 0 compact
  int conj = 0;                   // CWHAT='C'
  const int* mask = nullptr;      // device per-RHS flags (nonzero = compute)
  int nrhs = 1;
  // Optional, x-first pipeline only (conj = 0): the unconjugated FP64 sum
  // over compact sites of x*y of RHS r into dot_out[8*r + dot_k], reduced in
  // a fixed order inside the last MATVEC pass.  dot_part holds
  // nrhs * xdot_blocks(g) partials; dot_cnt one zeroed counter per RHS.
  double2* dot_out = nullptr;
  double2* dot_part = nullptr;
  unsigned* dot_cnt = nullptr;
  int dot_k = 0;
};

template <typename T> struct GreenArgs {
  int idipint = 0;
  double gamma = 0, pyd = 0, pzd = 0;
  double ak[3] = {0, 0, 0};
  double dx[3] = {1, 1, 1};
};

// The MATVEC engine for one prepared target (one Green tensor).
template <typename T> struct Engine {
  using C = cplx<T>;
  Geometry g;
  FftPlan px, py, pz;
  C *twx = nullptr, *twy = nullptr, *twz = nullptr;
  C* green = nullptr;
  int* occ = nullptr;      // [nat0]
  int* inv = nullptr;      // [nat], -1 for vacuum
  int16_t* iocc = nullptr; // [nat]
  int* rowq = nullptr;     // [nat/nx + 1]: occupied sites before each x row (row = iy + ny*iz)
  // MATVEC workspace
  C* zhat = nullptr;
  int zcap = 0;            // RHS capacity of zhat
  C* slab = nullptr;
  int slab_nr = 0, slab_B = 0;  // slab = slab_nr RHS x slab_B planes
  size_t slab_budget_elems = 0;
  int slices_layout = 0;
  int xpipe = 0;           // 1: x-first transposed pipeline (power-of-two grids)
  // launch shapes of the z-first pipeline (set from the environment at
  // prepare, changed by the autotuner): register-pass block sizes, y-pass
  // columns per block, complex elements per generic-pass tile (0: default)
  int tune_thz = 256, tune_thx = 256, tune_ly = 4, tune_tile = 0;
  // x-first z pass: 0 = three components per thread (kx_zg3, where it applies),
  // 1 = components exchanged through shared memory (kx_zg)
  int tune_zg = 0;
  // elements per RHS of the first-pass grid: the z-transformed grid (z-first)
  // or the x-transformed grid A (x-first)
  size_t zhat_per_rhs() const {
    return xpipe ? (size_t)3 * g.nz * g.Mx * g.ny : (size_t)3 * g.Mz * g.ny * g.nx;
  }
  cudaStream_t stream = 0;
  size_t bytes_allocated = 0;
  // device status word of the MATVEC kernels (0 = ok): a kernel whose bounded
  // wait for an asynchronous tile copy ran out sets it (matvec_check)
  int* d_err = nullptr;
  // tile moves of the FP32 256-point y passes by the tensor memory accelerator
  // (DDSCAT_B200_NOTMA=1 selects the per-thread copies)
  int use_tma = 1;
  // smallest RHS chunk per block for which the z pass stages its Green lines
  // in shared memory (kx_zg3r; DDSCAT_B200_ZG3R_MIN)
  int zg3r_min = 4;

  // pad: the Green tensor will be built here (build_green), so the FFT lengths
  // may be padded beyond 2n onto the register-FFT pipeline
  int init_geometry(int nx, int ny, int nz, int ipbc, int nat, int nat0, const int16_t* iocc_host, bool pad = false);
  int build_green(const GreenArgs<T>& ga);          // on-GPU direct sum + FFT to the octant
  int upload_green(const void* host_green);         // CPU-supplied CXZC (ddscat_cuda_prepare_f32)
  int interleave_green(const C* planar_dev);        // planar [6][P] -> green [P][6]
  int ensure_workspace(int nrhs);
  int matvec(const MvArgs<T>& a);
  void release();
};

// ---------------------------------------------------------------- vector kernels
template <typename T> struct VecOps {
  using C = cplx<T>;
  cudaStream_t stream = 0;
  double2* d_red = nullptr;    // reduction partials
  double2* d_out = nullptr;    // device results
  unsigned* d_count = nullptr; // last-block counters
  double2* h_out = nullptr;    // pinned host copy
  int nblocks = 0;
  int init(cudaStream_t s);
  void release();
  // results of up to 8 dots, each sum over conj(a)*b (conj=1) or a*b (conj=0)
  int dots(int n, int k, const C* const* a, const C* const* b, const int* conjf, double2* host_out);
  // the same products left in d_out[0..k) on the device (stream-ordered, no host copy)
  int dots_dev(int n, int k, const C* const* a, const C* const* b, const int* conjf);
  double2 dotc(int n, const C* a, const C* b, int* err);
  double2 dotu(int n, const C* a, const C* b, int* err);
  double nrm2(int n, const C* a, int* err);
  double norm_diff(int n, const C* a, const C* b, int* err);             // ||a-b||
  double norm_gap(int n, const C* a, const C* b, const C* c, int* err);  // ||a-b-c||
};

// elementwise launches (stream-ordered)
template <typename T> void v_copy(cplx<T>* d, const cplx<T>* a, int n, cudaStream_t s);
template <typename T> void v_zero(cplx<T>* d, int n, cudaStream_t s);
template <typename T> void v_diff(cplx<T>* d, const cplx<T>* a, const cplx<T>* b, int n, cudaStream_t s);  // d=a-b
// d = za*a + zb*b + zd*d   (any pointer may alias d; null a/b skip the term)
template <typename T>
void v_lincomb(cplx<T>* d, double2 zd, const cplx<T>* a, double2 za, const cplx<T>* b, double2 zb, int n, cudaStream_t s);
// d = a / adia_full[c*nat + occ[k]] (the DIAGL left preconditioner)
template <typename T>
void v_precon(cplx<T>* d, const cplx<T>* a, const cplx<T>* adia_full, const int* occ, int nat, int nat0, cudaStream_t s);
template <typename T> void v_gather(const cplx<T>* full, cplx<T>* compact, const int* occ, int nat, int nat0, cudaStream_t s);
template <typename T> void v_scatter(const cplx<T>* compact, cplx<T>* full, const int* occ, int nat, int nat0, cudaStream_t s);

// x-first transposed pipeline (matvec_x.cu)
template <typename T> bool xpipe_supported(const Geometry& g);
// smallest register-pipeline FFT length >= m for T (0 if none)
template <typename T> int xpipe_len(int m);
// Times the MATVEC of a prepared FP32 engine under the launch shapes that apply
// to its grid and keeps the fastest; default_ms / best_ms per call.
int autotune_engine(Engine<float>& e, int iters, float* default_ms, float* best_ms);
template <typename T> int matvec_xpipe(Engine<T>& E, const MvArgs<T>& a);
// whether the FP32 x-first pipeline has the components-per-thread z pass for length Mz
bool xzg3_supported(int Mz);
// partials per RHS of the fused x*y sum of the x-first pipeline (MvArgs::dot_out)
size_t xdot_blocks(const Geometry& g);
template <typename T> int interleave_green_zfast(Engine<T>& E, const cplx<T>* planar);
// 0, or 26 with the error text when a MATVEC kernel reported a timed-out tile
// copy since the last check (synchronises the engine's stream)
template <typename T> int matvec_check(Engine<T>& E);

}  // namespace ddb
