// Shared device/host helpers for the B200 DDA library.
//
// Complex numbers are plain float2 / double2 so that every buffer is a flat
// array of interleaved (re, im) pairs, exactly the cufftComplex /
// complex(c_float_complex) layout the DDSCAT Fortran caller passes
// (ddscat_cuda_unified/cuda/ddscat_matvec_cuda.h:11-51).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cmath>

#ifndef DDB_HD
#define DDB_HD __host__ __device__ __forceinline__
#endif

namespace ddb {

template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename C> DDB_HD C mk(double re, double im) { C c; c.x = re; c.y = im; return c; }
template <typename C, typename R> DDB_HD C mk2(R re, R im) { C c; c.x = re; c.y = im; return c; }
DDB_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
DDB_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
DDB_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
DDB_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
DDB_HD float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DDB_HD double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
DDB_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
DDB_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
DDB_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
DDB_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by i*s (s = +1 or -1 selects the sign of the rotation)
DDB_HD float2 cmuli(float2 a, float s) { return make_float2(-a.y * s, a.x * s); }

// Packed complex add / subtract: one Blackwell f32x2 instruction for both
// lanes (IEEE round-to-nearest per lane, identical results to two scalar
// adds).  Used by the FFT butterflies, where adds dominate; elsewhere the
// scalar forms are kept so the compiler can contract products into FMAs.
__device__ __forceinline__ float2 vadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 c;
  asm("add.rn.f32x2 %0, %1, %2;"
      : "=l"(reinterpret_cast<uint64_t&>(c))
      : "l"(reinterpret_cast<const uint64_t&>(a)), "l"(reinterpret_cast<const uint64_t&>(b)));
  return c;
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__device__ __forceinline__ float2 vsub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
  float2 c;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(reinterpret_cast<uint64_t&>(c))
      : "l"(reinterpret_cast<const uint64_t&>(a)), "l"(reinterpret_cast<const uint64_t&>(b)));
  return c;
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__device__ __forceinline__ double2 vadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 vsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// a + s*i*b and a - s*i*b (s = +-1): the rotated term stays scalar, where the
// swap and sign fold into the adds for free
template <int S, typename C> __device__ __forceinline__ C addrot(C a, C b) { return mk2<C>(a.x - S * b.y, a.y + S * b.x); }
template <int S, typename C> __device__ __forceinline__ C subrot(C a, C b) { return mk2<C>(a.x + S * b.y, a.y - S * b.x); }
DDB_HD double2 cmuli(double2 a, double s) { return make_double2(-a.y * s, a.x * s); }
DDB_HD double2 to_d(float2 a) { return make_double2((double)a.x, (double)a.y); }
DDB_HD double2 to_d(double2 a) { return a; }
template <typename C> DDB_HD C from_d(double2 a);
template <> DDB_HD float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> DDB_HD double2 from_d<double2>(double2 a) { return a; }
// complex-double scalar times vector element, evaluated in double then rounded
// to the vector type (the precision split of the Krylov updates)
DDB_HD float2 zmulv(double2 z, float2 v) {
  return make_float2((float)(z.x * (double)v.x - z.y * (double)v.y), (float)(z.x * (double)v.y + z.y * (double)v.x));
}
DDB_HD double2 zmulv(double2 z, double2 v) { return cmul(z, v); }
DDB_HD double2 zdiv(double2 a, double2 b) {
  double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
DDB_HD double zabs2(double2 a) { return a.x * a.x + a.y * a.y; }
DDB_HD bool zzero(double2 a) { return a.x == 0.0 && a.y == 0.0; }

inline size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

// Bulk global -> shared copies completed on a shared-memory mbarrier (sm_90+
// async proxy; no cluster multicast).  A CTA launched without a cluster is its
// own one-CTA cluster, so its shared::cta addresses are valid shared::cluster
// destinations.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one arrival that also announces `bytes` of transactions for the current phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// bytes and both addresses multiples of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Per-thread asynchronous 8-byte global -> shared copy (zero-fills when !ok;
// src must still be a valid address); completed by cp_async_wait_all.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(ok ? 8 : 0)
               : "memory");
}
// 16-byte form (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Wait for the phase of parity `par` to complete, at most `limit` polls;
// returns false if it did not complete in that time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t par, int limit) {
  const uint32_t a = smem_addr(bar);
  for (int k = 0; k < limit; ++k) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(par)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace ddb
