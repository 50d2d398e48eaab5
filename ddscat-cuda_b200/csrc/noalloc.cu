// MATVEC without any device allocation (library extension; no counterpart in
// the reference).
//
// Some callers cannot call cudaMalloc at the point where they need a MATVEC:
// real-time host loops that forbid allocation (and the device-wide
// synchronisation of cudaFree) once they have started, and applications that
// hand every byte of device memory to their own pool allocator and let no
// library allocate behind its back.  ddscat_b200_apply_noalloc_f32 serves
// them: it evaluates the same operator as ddscat_cuda_apply_f32 on
// caller-owned device vectors, and the FFT spectrum scratch of the MATVEC
// lives in the fixed array below instead of the engine's workspace.
//
// Limits and sharing:
//  * The scratch (48 MiB, 6,291,456 complex floats) must hold the
//    x-transformed grid and the half-padded spectrum of the prepared target:
//    3*nz*Mx*ny + 3*My*nz*Mx complex floats on the x-first pipeline, with
//    Mx, My the padded FFT lengths the prepare chose (2*nx, 2*ny, or the next
//    register-FFT length for a padded axis), 3*Mz*ny*nx + 3*ny*Mx*Mz on the
//    z-first one.  With M = 2n that is 18*NAT, so unpadded targets with
//    NAT = NX*NY*NZ <= 349,525 sites (e.g. 64^3) fit; padded grids need more
//    (72x72x64, NAT = 331,776, pads 144 to 192 and needs 9.7 M).  Targets
//    that do not fit are rejected with status 601 before any launch.
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
//  * The call must be made with the device that was current at prepare (the
//    prepared Green tensor and index tables live there); another current
//    device is rejected with status 600.
#include <atomic>
#include <cstddef>
#include "ddscat_b200.h"
#include "engine.h"

namespace ddb {

const Engine<float>* prepared_engine();
int prepared_device();

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)48 << 20;
constexpr size_t NOALLOC_SCRATCH_ELEMS = NOALLOC_SCRATCH_BYTES / sizeof(float2);
constexpr long long NOALLOC_MAX_NAT = (long long)(NOALLOC_SCRATCH_ELEMS / 18);

static __device__ __align__(256) float2 g_noalloc_scratch[NOALLOC_SCRATCH_ELEMS];

// device address of g_noalloc_scratch, looked up once per device (two host
// threads that race on the first lookup store the same address)
constexpr int NOALLOC_MAX_DEVICES = 64;
static std::atomic<float2*> g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

static int noalloc_scratch(int dev, float2** out) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) { set_error("apply_noalloc", "device ordinal out of range"); return 602; }
  float2* a = g_noalloc_addr[dev].load(std::memory_order_acquire);
  if (!a) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) { set_cuda_error("apply_noalloc: cudaGetSymbolAddress", e); return 602; }
    a = static_cast<float2*>(p);
    g_noalloc_addr[dev].store(a, std::memory_order_release);
  }
  *out = a;
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
  int dev = -1;
  const cudaError_t ge = cudaGetDevice(&dev);
  if (ge != cudaSuccess) { set_cuda_error("apply_noalloc: cudaGetDevice", ge); return 602; }
  if (dev != prepared_device()) {
    set_error("apply_noalloc", "the current device is not the one the target was prepared on");
    return 600;
  }
  if ((long long)prep->g.nat > NOALLOC_MAX_NAT) {
    char msg[200];
    std::snprintf(msg, sizeof(msg), "target has NAT=%d lattice sites; the fixed scratch (48 MiB) holds at most %lld",
                  prep->g.nat, NOALLOC_MAX_NAT);
    set_error("apply_noalloc", msg);
    return 601;
  }
  float2* scratch = nullptr;
  int rc = noalloc_scratch(dev, &scratch);
  if (rc) return rc;
  // A shallow copy of the prepared engine whose workspace is the fixed array:
  // one RHS, every middle-stage plane in one batch.
  Engine<float> e = *prep;
  const size_t za = e.zhat_per_rhs();
  const size_t sb = e.xpipe ? (size_t)3 * e.g.My * e.g.nz * e.g.Mx : (size_t)3 * e.g.ny * e.g.Mx * e.g.Mz;
  if (za + sb > (size_t)NOALLOC_SCRATCH_ELEMS) {
    char msg[240];
    std::snprintf(msg, sizeof(msg),
                  "the padded FFT grid of this target needs %zu complex floats of scratch; the fixed scratch (48 MiB) "
                  "holds at most %zu",
                  za + sb, (size_t)NOALLOC_SCRATCH_ELEMS);
    set_error("apply_noalloc", msg);
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
