// MATVEC without any device allocation (library extension; no counterpart in
// the reference).
//
// Some callers cannot call cudaMalloc at the point where they need a MATVEC:
// code being recorded into a CUDA graph by stream capture (cudaMalloc and
// cudaFree are not capturable, and cudaFree synchronises the whole device),
// real-time host loops that forbid allocation after start-up, and
// applications that hand every byte of device memory to their own pool.
// ddscat_b200_apply_noalloc_f32 serves them: it evaluates the same operator
// as ddscat_cuda_apply_f32 on caller-owned device vectors, and the FFT
// spectrum scratch of the MATVEC lives in the fixed array below instead of the
// engine's workspace.
//
// Limits and sharing:
//  * The scratch holds 18*NAT complex floats (the x-transformed grid, 6*NAT,
//    plus the half-padded spectrum, 12*NAT), so targets with
//    NAT = NX*NY*NZ <= NOALLOC_MAX_NAT (349,525 sites, e.g. 64^3) are
//    accepted; larger ones are rejected with status 601.
//  * The array is part of the library's device image: every GPU that loads
//    the library holds these 48 MiB until the process exits.
//  * Every call on a device uses the same array and it keeps the last call's
//    contents.  Nothing in it needs to start at zero: each pass writes every
//    element it later reads.  Calls whose work overlaps on the GPU (two
//    streams, two host threads) race on the array; serialise them.
//  * The first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (which may load the library's device code) and the
//    first call after each prepare registers the MATVEC kernels' shared-memory
//    limits; make those first calls before any stream capture.  After that a
//    call allocates nothing and only launches kernels on `stream`.
#include <cstddef>
#include "ddscat_b200.h"
#include "engine.h"

namespace ddb {

const Engine<float>* prepared_engine();

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)48 << 20;
constexpr size_t NOALLOC_SCRATCH_ELEMS = NOALLOC_SCRATCH_BYTES / sizeof(float2);
constexpr long long NOALLOC_MAX_NAT = (long long)(NOALLOC_SCRATCH_ELEMS / 18);

static __device__ __align__(256) float2 g_noalloc_scratch[NOALLOC_SCRATCH_ELEMS];

// device address of g_noalloc_scratch, looked up once per device
constexpr int NOALLOC_MAX_DEVICES = 64;
static float2* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};

static int noalloc_scratch(float2** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { set_cuda_error("apply_noalloc: cudaGetDevice", e); return 602; }
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) { set_error("apply_noalloc", "device ordinal out of range"); return 602; }
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) { set_cuda_error("apply_noalloc: cudaGetSymbolAddress", e); return 602; }
    g_noalloc_addr[dev] = static_cast<float2*>(p);
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

}  // namespace ddb

using namespace ddb;

extern "C" DDSCAT_CUDA_API int ddscat_b200_apply_noalloc_f32(int cwhat, const void* x, void* y, const void* adia,
                                                             const void* aoff, void* stream) {
  clear_error();
  const Engine<float>* prep = prepared_engine();
  if (!prep) { set_error("apply_noalloc", "not prepared"); return 600; }
  if ((cwhat != 'N' && cwhat != 'C') || !x || !y || !adia) { set_error("apply_noalloc", "invalid argument"); return 600; }
  if ((long long)prep->g.nat > NOALLOC_MAX_NAT) {
    char msg[200];
    std::snprintf(msg, sizeof(msg), "target has NAT=%d lattice sites; the fixed scratch (48 MiB) holds at most %lld",
                  prep->g.nat, NOALLOC_MAX_NAT);
    set_error("apply_noalloc", msg);
    return 601;
  }
  float2* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  // A shallow copy of the prepared engine whose workspace is the fixed array:
  // one RHS, every middle-stage plane in one batch.
  Engine<float> e = *prep;
  const size_t za = e.zhat_per_rhs();
  const size_t sb = e.xpipe ? (size_t)3 * e.g.My * e.g.nz * e.g.Mx : (size_t)3 * e.g.ny * e.g.Mx * e.g.Mz;
  if (za + sb > (size_t)NOALLOC_SCRATCH_ELEMS) {
    set_error("apply_noalloc", "the padded FFT grid of this target does not fit the fixed scratch (48 MiB)");
    return 601;
  }
  e.zhat = scratch;
  e.zcap = 1;
  e.slab = scratch + za;
  e.slab_nr = 1;
  e.slab_B = e.xpipe ? e.g.Mx : e.g.Mz;
  e.stream = static_cast<cudaStream_t>(stream);
  MvArgs<float> a;
  a.x = static_cast<const float2*>(x);
  a.y = static_cast<float2*>(y);
  a.io_full = 1;
  a.adia = static_cast<const float2*>(adia);
  a.aoff = static_cast<const float2*>(aoff);
  a.a_full = 1;
  a.conj = (cwhat == 'C');
  a.nrhs = 1;
  return e.matvec(a);
}
