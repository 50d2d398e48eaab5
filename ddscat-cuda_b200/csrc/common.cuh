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

}  // namespace ddb
