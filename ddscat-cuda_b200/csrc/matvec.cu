// FFT-accelerated DDA MATVEC, z-first pipeline (sm_100a).
//
// y = CXADIA o x - (G * x) + CXAOFF 3x3 site blocks, unoccupied sites zeroed;
// CWHAT='C' conjugates x on input and y on output.  This is the operator of
// ddscat_cuda_unified/fortran/cprod_cuda.f90:446-607 evaluated as in
// ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu:104-118 (pad, FFT(+i), Green
// 3x3 multiply from the octant with sign flips, FFT(-i), finish with 1/ngrid),
// but organised per axis so the zero-padded half is never transformed on the
// forward side and never produced on the inverse side:
//   k_zfwd    : compact/full x -> z-FFT(+i) of n_z inputs -> zhat (M_z planes)
//   k_xfwd    : zhat plane rows (n_x inputs) -> x-FFT(+i) -> slab rows (M_x)
//   k_ygreen  : slab columns (n_y inputs) -> y-FFT(+i) -> Green -> y-FFT(-i),
//               keep n_y outputs
//   k_xinv    : slab rows -> x-FFT(-i), keep n_x -> zhat
//   k_zinv_fin: zhat columns -> z-FFT(-i), keep n_z -> finish -> y
#include <algorithm>
#include <cstdlib>
#include "engine.h"
#include "fftreg.cuh"

namespace ddb {

template <typename T> struct MvParams {
  int nx, ny, nz, Mx, My, Mz, nat, nat0;
  const cplx<T>* x;
  size_t x_rs;
  cplx<T>* y;
  size_t y_rs;
  const cplx<T>* adia;
  const cplx<T>* aoff;
  size_t a_rs;
  int io_full, a_full, conj;
  const int* inv;
  const int16_t* iocc;
  const int* mask;
  int rhs0;  // global index of local RHS 0 (for the mask)
  cplx<T>* zhat;
  size_t zhat_rs;
  cplx<T>* slab;
  int kz0, nplanes;  // planes kz0 .. kz0+nplanes-1 live in the slab
  int slab_rhs0;     // local RHS index of slab RHS 0 (relative to zhat)
  const cplx<T>* green;
  int ipbc;
  FftPlan px, py, pz;
  const cplx<T>* twx;
  const cplx<T>* twy;
  const cplx<T>* twz;
  int tz, ry, ty;  // tile widths
  int lsz, lsx, lsy;  // register-path line strides (complex elements)
  T inv_ngrid;
};

template <typename T> __device__ __forceinline__ bool rhs_off(const MvParams<T>& P, int rl) {
  return P.mask != nullptr && P.mask[P.rhs0 + rl] == 0;
}

// ---------------------------------------------------------------- z forward
template <typename T> __global__ void __launch_bounds__(256) k_zfwd(MvParams<T> P) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TX = P.tz;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + (size_t)TX * P.Mz;
  const int ix0 = blockIdx.x * TX, iy = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z % 3;
  if (rhs_off(P, rl)) return;
  const C* x = P.x + (size_t)rl * P.x_rs;
  const size_t S = P.io_full ? (size_t)P.nat : (size_t)P.nat0;
  const int tot = TX * P.Mz;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int l = t % TX, e = t / TX, ix = ix0 + l;
    C v = mk<C>(0, 0);
    if (e < P.nz && ix < P.nx) {
      const size_t j = (size_t)ix + (size_t)P.nx * ((size_t)iy + (size_t)P.ny * e);
      if (P.io_full) {
        v = x[c * S + j];
      } else {
        const int q = P.inv[j];
        if (q >= 0) v = x[c * S + q];
      }
      if (P.conj) v.y = -v.y;
    }
    A[e * TX + l] = v;
  }
  __syncthreads();
  C* R = fft_tile<+1>(A, B, Lay{1, TX}, TX, P.pz, P.twz);
  C* zh = P.zhat + (size_t)rl * P.zhat_rs + (size_t)c * P.Mz * P.ny * P.nx;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int l = t % TX, e = t / TX, ix = ix0 + l;
    if (ix < P.nx) zh[((size_t)e * P.ny + iy) * P.nx + ix] = R[e * TX + l];
  }
}

// ---------------------------------------------------------------- x forward
template <typename T> __global__ void __launch_bounds__(256) k_xfwd(MvParams<T> P) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int RY = P.ry, LD = P.Mx + 1;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + (size_t)RY * LD;
  const int iy0 = blockIdx.x * RY, kzl = blockIdx.y, kz = P.kz0 + kzl;
  const int rs = blockIdx.z / 3, c = blockIdx.z % 3, rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  const C* zh = P.zhat + (size_t)rl * P.zhat_rs + ((size_t)c * P.Mz + kz) * P.ny * P.nx;
  const int tot = RY * P.Mx;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int e = t % P.Mx, l = t / P.Mx, iy = iy0 + l;
    C v = mk<C>(0, 0);
    if (e < P.nx && iy < P.ny) v = zh[(size_t)iy * P.nx + e];
    A[l * LD + e] = v;
  }
  __syncthreads();
  C* R = fft_tile<+1>(A, B, Lay{LD, 1}, RY, P.px, P.twx);
  C* sl = P.slab + (((size_t)rs * 3 + c) * P.nplanes + kzl) * P.ny * P.Mx;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int e = t % P.Mx, l = t / P.Mx, iy = iy0 + l;
    if (iy < P.ny) sl[(size_t)iy * P.Mx + e] = R[l * LD + e];
  }
}

// Green tensor at spectral point (kx,ky,kz): symmetric 3x3 (a11,a12,a13,a22,a23,a33)
template <typename T>
__device__ __forceinline__ void green_at(const MvParams<T>& P, int kx, int ky, int kz, cplx<T> a[6]) {
  // Green storage is point-interleaved: g[point*6 + m], m = (xx,xy,xz,yy,yz,zz)
  size_t b;
  T sxy = (T)1, sxz = (T)1, syz = (T)1;
  if (P.ipbc == 0) {
    const T sx = 2 * kx <= P.Mx ? (T)1 : (T)-1, sy = 2 * ky <= P.My ? (T)1 : (T)-1, sz = 2 * kz <= P.Mz ? (T)1 : (T)-1;
    const int irx = min(kx, P.Mx - kx), iry = min(ky, P.My - ky), irz = min(kz, P.Mz - kz);
    b = (size_t)irx + (size_t)(P.Mx / 2 + 1) * ((size_t)iry + (size_t)(P.My / 2 + 1) * irz);
    sxy = sx * sy; sxz = sx * sz; syz = sy * sz;
  } else {
    b = (size_t)kx + (size_t)P.Mx * ((size_t)ky + (size_t)P.My * kz);
  }
  const cplx<T>* gp = P.green + 6 * b;
  if constexpr (sizeof(cplx<T>) == 8) {
    const float4* g4 = reinterpret_cast<const float4*>(gp);  // 48-byte point record, 16-byte aligned
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const float4 q = __ldg(g4 + m);
      a[2 * m] = mk<cplx<T>>(q.x, q.y);
      a[2 * m + 1] = mk<cplx<T>>(q.z, q.w);
    }
  } else {
#pragma unroll
    for (int m = 0; m < 6; ++m) a[m] = gp[m];
  }
  a[1] = cscale(a[1], sxy);
  a[2] = cscale(a[2], sxz);
  a[4] = cscale(a[4], syz);
}

// ---------------------------------------------------------------- y forward * Green * y inverse
template <typename T> __global__ void __launch_bounds__(256) k_ygreen(MvParams<T> P) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TX = P.ty, My = P.My;
  C* D = reinterpret_cast<C*>(smem_raw);  // [3][My][TX]
  C* S = D + (size_t)3 * My * TX;         // scratch [My][TX]
  const int kx0 = blockIdx.x * TX, kzl = blockIdx.y, kz = P.kz0 + kzl;
  const int rs = blockIdx.z, rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  const size_t plane = (size_t)P.ny * P.Mx;
  C* sl0 = P.slab + ((size_t)rs * 3 * P.nplanes + kzl) * plane;
  const size_t cstride = (size_t)P.nplanes * plane;
  const int tot = TX * My;
  for (int t = threadIdx.x; t < 3 * tot; t += blockDim.x) {
    const int c = t / tot, u = t % tot, l = u % TX, e = u / TX, kx = kx0 + l;
    C v = mk<C>(0, 0);
    if (e < P.ny && kx < P.Mx) v = sl0[c * cstride + (size_t)e * P.Mx + kx];
    D[(size_t)c * tot + u] = v;
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    C* Dc = D + (size_t)c * tot;
    C* R = fft_tile<+1>(Dc, S, Lay{1, TX}, TX, P.py, P.twy);
    if (R != Dc) {
      for (int u = threadIdx.x; u < tot; u += blockDim.x) Dc[u] = R[u];
      __syncthreads();
    }
  }
  for (int u = threadIdx.x; u < tot; u += blockDim.x) {
    const int l = u % TX, ky = u / TX, kx = kx0 + l;
    if (kx >= P.Mx) continue;
    C a[6];
    green_at(P, kx, ky, kz, a);
    const C px = D[u], py = D[tot + u], pz = D[2 * tot + u];
    D[u] = cadd(cadd(cmul(a[0], px), cmul(a[1], py)), cmul(a[2], pz));
    D[tot + u] = cadd(cadd(cmul(a[1], px), cmul(a[3], py)), cmul(a[4], pz));
    D[2 * tot + u] = cadd(cadd(cmul(a[2], px), cmul(a[4], py)), cmul(a[5], pz));
  }
  __syncthreads();
  for (int c = 0; c < 3; ++c) {
    C* Dc = D + (size_t)c * tot;
    C* R = fft_tile<-1>(Dc, S, Lay{1, TX}, TX, P.py, P.twy);
    if (R != Dc) {
      for (int u = threadIdx.x; u < tot; u += blockDim.x) Dc[u] = R[u];
      __syncthreads();
    }
  }
  const int totn = TX * P.ny;
  for (int t = threadIdx.x; t < 3 * totn; t += blockDim.x) {
    const int c = t / totn, u = t % totn, l = u % TX, e = u / TX, kx = kx0 + l;
    if (kx < P.Mx) sl0[c * cstride + (size_t)e * P.Mx + kx] = D[(size_t)c * tot + u];
  }
}

// ---------------------------------------------------------------- x inverse
template <typename T> __global__ void __launch_bounds__(256) k_xinv(MvParams<T> P) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int RY = P.ry, LD = P.Mx + 1;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + (size_t)RY * LD;
  const int iy0 = blockIdx.x * RY, kzl = blockIdx.y, kz = P.kz0 + kzl;
  const int rs = blockIdx.z / 3, c = blockIdx.z % 3, rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  const C* sl = P.slab + (((size_t)rs * 3 + c) * P.nplanes + kzl) * P.ny * P.Mx;
  const int tot = RY * P.Mx;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int e = t % P.Mx, l = t / P.Mx, iy = iy0 + l;
    C v = mk<C>(0, 0);
    if (iy < P.ny) v = sl[(size_t)iy * P.Mx + e];
    A[l * LD + e] = v;
  }
  __syncthreads();
  C* R = fft_tile<-1>(A, B, Lay{LD, 1}, RY, P.px, P.twx);
  C* zh = P.zhat + (size_t)rl * P.zhat_rs + ((size_t)c * P.Mz + kz) * P.ny * P.nx;
  const int totn = RY * P.nx;
  for (int t = threadIdx.x; t < totn; t += blockDim.x) {
    const int e = t % P.nx, l = t / P.nx, iy = iy0 + l;
    if (iy < P.ny) zh[(size_t)iy * P.nx + e] = R[l * LD + e];
  }
}

// ---------------------------------------------------------------- z inverse + finish
template <typename T> __global__ void __launch_bounds__(256) k_zinv_fin(MvParams<T> P) {
  using C = cplx<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int TX = P.tz;
  C* A = reinterpret_cast<C*>(smem_raw);
  C* B = A + (size_t)TX * P.Mz;
  const int ix0 = blockIdx.x * TX, iy = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z % 3;
  if (rhs_off(P, rl)) return;
  const C* zh = P.zhat + (size_t)rl * P.zhat_rs + (size_t)c * P.Mz * P.ny * P.nx;
  const int tot = TX * P.Mz;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int l = t % TX, e = t / TX, ix = ix0 + l;
    C v = mk<C>(0, 0);
    if (ix < P.nx) v = zh[((size_t)e * P.ny + iy) * P.nx + ix];
    A[e * TX + l] = v;
  }
  __syncthreads();
  C* R = fft_tile<-1>(A, B, Lay{1, TX}, TX, P.pz, P.twz);
  const C* x = P.x + (size_t)rl * P.x_rs;
  C* y = P.y + (size_t)rl * P.y_rs;
  const C* ad = P.adia + (size_t)rl * P.a_rs;
  const C* ao = P.aoff ? P.aoff + (size_t)rl * P.a_rs : nullptr;
  const size_t S = P.io_full ? (size_t)P.nat : (size_t)P.nat0;
  const size_t SA = P.a_full ? (size_t)P.nat : (size_t)P.nat0;
  const int totn = TX * P.nz;
  for (int t = threadIdx.x; t < totn; t += blockDim.x) {
    const int l = t % TX, iz = t / TX, ix = ix0 + l;
    if (ix >= P.nx) continue;
    const size_t j = (size_t)ix + (size_t)P.nx * ((size_t)iy + (size_t)P.ny * iz);
    size_t q;
    if (P.io_full) {
      q = j;
      if (P.iocc[j] == 0) { y[c * S + q] = mk<C>(0, 0); continue; }
    } else {
      const int qq = P.inv[j];
      if (qq < 0) continue;
      q = (size_t)qq;
    }
    const size_t qa = P.a_full ? j : q;
    C xc = x[c * S + q];
    if (P.conj) xc.y = -xc.y;
    C w = cscale(R[iz * TX + l], P.inv_ngrid);
    C yv = csub(cmul(ad[c * SA + qa], xc), w);
    if (ao) {
      C x1 = x[q], x2 = x[S + q], x3 = x[2 * S + q];
      if (P.conj) { x1.y = -x1.y; x2.y = -x2.y; x3.y = -x3.y; }
      const C a23 = ao[qa], a31 = ao[SA + qa], a12 = ao[2 * SA + qa];
      if (c == 0) yv = cadd(yv, cadd(cmul(a31, x3), cmul(a12, x2)));
      else if (c == 1) yv = cadd(yv, cadd(cmul(a12, x1), cmul(a23, x3)));
      else yv = cadd(yv, cadd(cmul(a23, x2), cmul(a31, x1)));
    }
    if (P.conj) yv.y = -yv.y;
    y[c * S + q] = yv;
  }
}


// ================================================================ register path
// Power-of-two axis lengths 16..512 use register-resident line transforms
// (fftreg.cuh): each pass is one coalesced global read, one shared-memory
// transpose per transform and one coalesced global write.  Column passes put
// L = blockDim/T adjacent columns in the fast thread index (coalescing along
// the contiguous axis); row passes put the T threads of a row adjacent.

template <typename T>
__device__ __forceinline__ void finish_site(const MvParams<T>& P, int rl, int c, int ix, int iy, int iz, cplx<T> wraw) {
  using C = cplx<T>;
  const C* x = P.x + (size_t)rl * P.x_rs;
  C* y = P.y + (size_t)rl * P.y_rs;
  const C* ad = P.adia + (size_t)rl * P.a_rs;
  const C* ao = P.aoff ? P.aoff + (size_t)rl * P.a_rs : nullptr;
  const size_t S = P.io_full ? (size_t)P.nat : (size_t)P.nat0;
  const size_t SA = P.a_full ? (size_t)P.nat : (size_t)P.nat0;
  const size_t j = (size_t)ix + (size_t)P.nx * ((size_t)iy + (size_t)P.ny * iz);
  size_t q;
  if (P.io_full) {
    q = j;
    if (P.iocc[j] == 0) { y[c * S + q] = mk<C>(0, 0); return; }
  } else {
    const int qq = P.inv[j];
    if (qq < 0) return;
    q = (size_t)qq;
  }
  const size_t qa = P.a_full ? j : q;
  C xc = x[c * S + q];
  if (P.conj) xc.y = -xc.y;
  const C w = cscale(wraw, P.inv_ngrid);
  C yv = csub(cmul(ad[c * SA + qa], xc), w);
  if (ao) {
    C x1 = x[q], x2 = x[S + q], x3 = x[2 * S + q];
    if (P.conj) { x1.y = -x1.y; x2.y = -x2.y; x3.y = -x3.y; }
    const C a23 = ao[qa], a31 = ao[SA + qa], a12 = ao[2 * SA + qa];
    if (c == 0) yv = cadd(yv, cadd(cmul(a31, x3), cmul(a12, x2)));
    else if (c == 1) yv = cadd(yv, cadd(cmul(a12, x1), cmul(a23, x3)));
    else yv = cadd(yv, cadd(cmul(a23, x2), cmul(a31, x1)));
  }
  if (P.conj) yv.y = -yv.y;
  y[c * S + q] = yv;
}

template <typename T, int N> __global__ void __launch_bounds__(256) k_zfwd_r(MvParams<T> P) {
  using C = cplx<T>;
  constexpr int E = RegShape<N>::E, TT = RegShape<N>::T;
  const int LS = P.lsz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  C* tws = sm + (size_t)(blockDim.x / TT) * LS;  // N twiddles after the line scratches
  const int L = blockDim.x / TT, l = threadIdx.x % L, t = threadIdx.x / L;
  const int ix = blockIdx.x * L + l, iy = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z % 3;
  if (rhs_off(P, rl)) return;
  for (int u = threadIdx.x; u < N; u += blockDim.x) tws[u] = P.twz[u];
  __syncthreads();
  const C* x = P.x + (size_t)rl * P.x_rs;
  const size_t S = P.io_full ? (size_t)P.nat : (size_t)P.nat0;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int iz = t + TT * i;
    v[i] = mk<C>(0, 0);
    if (iz < P.nz && ix < P.nx) {
      const size_t j = (size_t)ix + (size_t)P.nx * ((size_t)iy + (size_t)P.ny * iz);
      if (P.io_full) {
        v[i] = x[c * S + j];
      } else {
        const int q = P.inv[j];
        if (q >= 0) v[i] = x[c * S + q];
      }
      if (P.conj) v[i].y = -v[i].y;
    }
  }
  line_fft<E, TT, +1, true>(v, sm + l * LS, t, tws);
  if (ix < P.nx) {
    C* zh = P.zhat + (size_t)rl * P.zhat_rs + (size_t)c * P.Mz * P.ny * P.nx + (size_t)iy * P.nx + ix;
#pragma unroll
    for (int i = 0; i < E; ++i) zh[(size_t)(t + TT * i) * P.ny * P.nx] = v[i];
  }
}

template <typename T, int N> __global__ void __launch_bounds__(256) k_xfwd_r(MvParams<T> P) {
  using C = cplx<T>;
  constexpr int E = RegShape<N>::E, TT = RegShape<N>::T;
  const int LS = P.lsx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  C* tws = sm + (size_t)(blockDim.x / TT) * LS;  // N twiddles after the line scratches
  const int RL = blockDim.x / TT, t = threadIdx.x % TT, l = threadIdx.x / TT;
  const int iy = blockIdx.x * RL + l, kzl = blockIdx.y, kz = P.kz0 + kzl;
  const int rs = blockIdx.z / 3, c = blockIdx.z % 3, rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  for (int u = threadIdx.x; u < N; u += blockDim.x) tws[u] = P.twx[u];
  __syncthreads();
  const C* zh = P.zhat + (size_t)rl * P.zhat_rs + ((size_t)c * P.Mz + kz) * P.ny * P.nx + (size_t)iy * P.nx;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int ix = t + TT * i;
    v[i] = (ix < P.nx && iy < P.ny) ? zh[ix] : mk<C>(0, 0);
  }
  line_fft<E, TT, +1, false>(v, sm + l * LS, t, tws);
  if (iy < P.ny) {
    C* sl = P.slab + (((size_t)rs * 3 + c) * P.nplanes + kzl) * P.ny * P.Mx + (size_t)iy * P.Mx;
#pragma unroll
    for (int i = 0; i < E; ++i) sl[t + TT * i] = v[i];
  }
}

template <typename T, int N> __global__ void __launch_bounds__(384) k_ygreen_r(MvParams<T> P) {
  // Thread (l, t, c): column l of the block's L columns, line thread t, field
  // component c.  (1) forward y-FFT of every component's column into its line
  // region (the same region serves as the transpose scratch), (2) Green 3x3
  // multiply with one thread per spectral point, (3) inverse y-FFTs, truncated
  // store.  Grid: x = RHS (so consecutive blocks share the Green tile in L2),
  // y = column tile, z = plane.
  using C = cplx<T>;
  constexpr int E = RegShape<N>::E, TT = RegShape<N>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int LS = P.lsy;
  const int L = blockDim.x / (3 * TT);
  const int l = threadIdx.x % L, t = (threadIdx.x / L) % TT, c = threadIdx.x / (L * TT);
  C* tws = reinterpret_cast<C*>(smem_raw);  // N twiddles
  C* lines = tws + N;                        // [3][L][LS]
  C* my = lines + (size_t)(c * L + l) * LS;
  for (int u = threadIdx.x; u < N; u += blockDim.x) tws[u] = P.twy[u];
  const int rs = blockIdx.x, kx0 = blockIdx.y * L, kx = kx0 + l, kzl = blockIdx.z, kz = P.kz0 + kzl;
  const int rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  __syncthreads();
  const size_t plane = (size_t)P.ny * P.Mx, cstride = (size_t)P.nplanes * plane;
  C* col = P.slab + ((size_t)rs * 3 * P.nplanes + kzl) * plane + c * cstride + kx;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int iy = t + TT * i;
    v[i] = (iy < P.ny && kx < P.Mx) ? col[(size_t)iy * P.Mx] : mk<C>(0, 0);
  }
  line_fft<E, TT, +1, true>(v, my, t, tws);
#pragma unroll
  for (int i = 0; i < E; ++i) my[t + TT * i] = v[i];
  __syncthreads();
  for (int u = threadIdx.x; u < N * L; u += blockDim.x) {
    const int ll = u % L, ky = u / L, kxx = kx0 + ll;
    if (kxx >= P.Mx) continue;
    C a[6];
    green_at(P, kxx, ky, kz, a);
    C* p0 = lines + (size_t)ll * LS + ky;
    C* p1 = p0 + (size_t)L * LS;
    C* p2 = p1 + (size_t)L * LS;
    const C px = *p0, py = *p1, pz = *p2;
    *p0 = cadd(cadd(cmul(a[0], px), cmul(a[1], py)), cmul(a[2], pz));
    *p1 = cadd(cadd(cmul(a[1], px), cmul(a[3], py)), cmul(a[4], pz));
    *p2 = cadd(cadd(cmul(a[2], px), cmul(a[4], py)), cmul(a[5], pz));
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < E; ++i) v[i] = my[t + TT * i];
  __syncthreads();  // the region is reused as transpose scratch below
  line_fft<E, TT, -1, true>(v, my, t, tws);
  if (kx < P.Mx) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int iy = t + TT * i;
      if (iy < P.ny) col[(size_t)iy * P.Mx] = v[i];
    }
  }
}

template <typename T, int N> __global__ void __launch_bounds__(256) k_xinv_r(MvParams<T> P) {
  using C = cplx<T>;
  constexpr int E = RegShape<N>::E, TT = RegShape<N>::T;
  const int LS = P.lsx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  C* tws = sm + (size_t)(blockDim.x / TT) * LS;  // N twiddles after the line scratches
  const int RL = blockDim.x / TT, t = threadIdx.x % TT, l = threadIdx.x / TT;
  const int iy = blockIdx.x * RL + l, kzl = blockIdx.y, kz = P.kz0 + kzl;
  const int rs = blockIdx.z / 3, c = blockIdx.z % 3, rl = P.slab_rhs0 + rs;
  if (rhs_off(P, rl)) return;
  for (int u = threadIdx.x; u < N; u += blockDim.x) tws[u] = P.twx[u];
  __syncthreads();
  const C* sl = P.slab + (((size_t)rs * 3 + c) * P.nplanes + kzl) * P.ny * P.Mx + (size_t)iy * P.Mx;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) v[i] = (iy < P.ny) ? sl[t + TT * i] : mk<C>(0, 0);
  line_fft<E, TT, -1, false>(v, sm + l * LS, t, tws);
  if (iy < P.ny) {
    C* zh = P.zhat + (size_t)rl * P.zhat_rs + ((size_t)c * P.Mz + kz) * P.ny * P.nx + (size_t)iy * P.nx;
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int ix = t + TT * i;
      if (ix < P.nx) zh[ix] = v[i];
    }
  }
}

template <typename T, int N> __global__ void __launch_bounds__(256) k_zinv_fin_r(MvParams<T> P) {
  using C = cplx<T>;
  constexpr int E = RegShape<N>::E, TT = RegShape<N>::T;
  const int LS = P.lsz;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  C* tws = sm + (size_t)(blockDim.x / TT) * LS;  // N twiddles after the line scratches
  const int L = blockDim.x / TT, l = threadIdx.x % L, t = threadIdx.x / L;
  const int ix = blockIdx.x * L + l, iy = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z % 3;
  if (rhs_off(P, rl)) return;
  for (int u = threadIdx.x; u < N; u += blockDim.x) tws[u] = P.twz[u];
  __syncthreads();
  const C* zh = P.zhat + (size_t)rl * P.zhat_rs + (size_t)c * P.Mz * P.ny * P.nx + (size_t)iy * P.nx + ix;
  C v[E];
#pragma unroll
  for (int i = 0; i < E; ++i) v[i] = (ix < P.nx) ? zh[(size_t)(t + TT * i) * P.ny * P.nx] : mk<C>(0, 0);
  line_fft<E, TT, -1, true>(v, sm + l * LS, t, tws);
  if (ix < P.nx) {
#pragma unroll
    for (int i = 0; i < E; ++i) {
      const int iz = t + TT * i;
      if (iz < P.nz) finish_site(P, rl, c, ix, iy, iz, v[i]);
    }
  }
}

enum class Pass { ZF, XF, YG, XI, ZI };

template <typename T, int N> static const void* reg_kernel(Pass p) {
  switch (p) {
    case Pass::ZF: return (const void*)k_zfwd_r<T, N>;
    case Pass::XF: return (const void*)k_xfwd_r<T, N>;
    case Pass::YG: return (const void*)k_ygreen_r<T, N>;
    case Pass::XI: return (const void*)k_xinv_r<T, N>;
    default: return (const void*)k_zinv_fin_r<T, N>;
  }
}

// Register kernel for this pass and axis length, or null (generic path).
template <typename T> static const void* pick_reg(Pass p, int n) {
  if (env_flag("DDSCAT_B200_GENERIC_FFT")) return nullptr;
  if (sizeof(T) == 8) return nullptr;  // FP64 engine: generic path (register budget)
  if (p == Pass::YG && n == 512) return nullptr;
  switch (n) {
    case 16: return reg_kernel<T, 16>(p);
    case 32: return reg_kernel<T, 32>(p);
    case 64: return reg_kernel<T, 64>(p);
    case 128: return reg_kernel<T, 128>(p);
    case 256: return reg_kernel<T, 256>(p);
    case 512: return reg_kernel<T, 512>(p);
    default: return nullptr;
  }
}

static int reg_T(int n) { return n <= 32 ? 4 : (n <= 128 ? 8 : 16); }
static int reg_E(int n) { return n / reg_T(n); }

template <typename T> static int launch_k(const void* f, dim3 g, int threads, size_t sm, cudaStream_t st, MvParams<T>& P) {
  void* args[] = {(void*)&P};
  note_launch();
  cudaError_t e = cudaLaunchKernel(f, g, dim3(threads), args, sm, st);
  if (e != cudaSuccess) { set_cuda_error("MATVEC launch", e); return 1; }
  return 0;
}

// ---------------------------------------------------------------- host side
static int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  return std::atoi(v);
}

template <typename T> static cplx<T>* upload_twiddles(int n, size_t& bytes) {
  std::vector<cplx<T>> h(n);
  const double pi = 3.14159265358979323846;
  for (int m = 0; m < n; ++m) {
    const double a = -2.0 * pi * (double)m / (double)n;
    h[m] = mk<cplx<T>>(std::cos(a), std::sin(a));
  }
  cplx<T>* d = nullptr;
  if (cudaMalloc((void**)&d, n * sizeof(cplx<T>)) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), n * sizeof(cplx<T>), cudaMemcpyHostToDevice);
  bytes += n * sizeof(cplx<T>);
  return d;
}

template <typename T>
int Engine<T>::init_geometry(int nx, int ny, int nz, int ipbc, int nat, int nat0, const int16_t* iocc_host, bool pad) {
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.Mx = 2 * nx; g.My = 2 * ny; g.Mz = 2 * nz;
  g.nat = nat; g.nat0 = nat0; g.ipbc = ipbc;
  if (pad && ipbc == 0 && nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && !env_flag("DDSCAT_B200_NOPAD") &&
      !xpipe_supported<T>(g)) {
    // pad to the register-FFT lengths when the padded grid has at most 2.5x the
    // points of the 2n grid (the register pipeline is ~4x faster per point);
    // even n only (the row passes move element pairs of 16 bytes)
    Geometry p = g;
    p.Mx = xpipe_len<T>(2 * nx); p.My = xpipe_len<T>(2 * ny); p.Mz = xpipe_len<T>(2 * nz);
    if (p.Mx && p.My && p.Mz && (double)p.ngrid() <= 2.5 * (double)g.ngrid() && xpipe_supported<T>(p)) g = p;
  }
  px = make_fft_plan(g.Mx);
  py = make_fft_plan(g.My);
  pz = make_fft_plan(g.Mz);
  xpipe = xpipe_supported<T>(g) ? 1 : 0;
  tune_thz = env_int("DDSCAT_B200_TH_Z", 256);
  tune_thx = env_int("DDSCAT_B200_TH_X", 256);
  tune_ly = std::max(1, env_int("DDSCAT_B200_LY", 4));
  tune_tile = env_int("DDSCAT_B200_TILE", 0);
  tune_zg = env_flag("DDSCAT_B200_ZG") ? 1 : 0;
  use_tma = env_flag("DDSCAT_B200_NOTMA") ? 0 : 1;
  zg3r_min = std::max(1, env_int("DDSCAT_B200_ZG3R_MIN", 4));
  if (!d_err) {
    if (cudaMalloc((void**)&d_err, sizeof(int)) != cudaSuccess) { set_error("prepare", "status word"); return 1; }
    cudaMemset(d_err, 0, sizeof(int));
  }
  if (px.nstages < 0 || py.nstages < 0 || pz.nstages < 0) {
    set_error("prepare", "FFT length has too many prime factors");
    return 1;
  }
  twx = upload_twiddles<T>(g.Mx, bytes_allocated);
  twy = upload_twiddles<T>(g.My, bytes_allocated);
  twz = upload_twiddles<T>(g.Mz, bytes_allocated);
  if (!twx || !twy || !twz) { set_error("prepare", "twiddle allocation failed"); return 1; }
  std::vector<int> occ_h, inv_h((size_t)nat, -1);
  occ_h.reserve(nat0);
  for (int j = 0; j < nat; ++j)
    if (iocc_host[j] != 0) { inv_h[j] = (int)occ_h.size(); occ_h.push_back(j); }
  if ((int)occ_h.size() != nat0) {
    char msg[160];
    std::snprintf(msg, sizeof(msg), "IOCC contains %zu occupied sites but NAT0=%d", occ_h.size(), nat0);
    set_error("occupied-index map", msg);
    return 2;
  }
  // compact index of the first occupied site of every x row: the sites of
  // consecutive rows occupy one contiguous compact range
  const int nrows = nat / nx;
  std::vector<int> rowq_h((size_t)nrows + 1, 0);
  for (int r = 0; r < nrows; ++r) {
    int c = 0;
    for (int ix = 0; ix < nx; ++ix) c += iocc_host[(size_t)r * nx + ix] != 0;
    rowq_h[r + 1] = rowq_h[r] + c;
  }
  cudaError_t e;
  e = cudaMalloc((void**)&occ, (size_t)nat0 * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&inv, (size_t)nat * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&iocc, (size_t)nat * sizeof(int16_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&rowq, ((size_t)nrows + 1) * sizeof(int));
  if (e != cudaSuccess) { set_cuda_error("prepare: index maps", e); return 3; }
  bytes_allocated += (size_t)nat0 * 4 + (size_t)nat * 6 + ((size_t)nrows + 1) * 4;
  cudaMemcpy(occ, occ_h.data(), (size_t)nat0 * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(inv, inv_h.data(), (size_t)nat * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemcpy(rowq, rowq_h.data(), ((size_t)nrows + 1) * sizeof(int), cudaMemcpyHostToDevice);
  e = cudaMemcpy(iocc, iocc_host, (size_t)nat * sizeof(int16_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { set_cuda_error("prepare: index map H2D", e); return 3; }
  e = cudaMalloc((void**)&green, g.green_count() * sizeof(C));
  if (e != cudaSuccess) { set_cuda_error("malloc resident Green", e); return 4; }
  bytes_allocated += g.green_count() * sizeof(C);
  // slab budget: FFT3D keeps the xy spectrum of all kz planes of up to 4 GiB
  // worth of RHS per batch (one Green pass per batch); SLICES keeps 4 planes.
  const int mb = env_int("DDSCAT_B200_SLAB_MB", 4096);
  slab_budget_elems = (size_t)mb * 1024 * 1024 / sizeof(C);
  return 0;
}

template <typename T> int Engine<T>::ensure_workspace(int nrhs) {
  const size_t per_rhs_z = zhat_per_rhs();
  // one middle-stage plane, 3 comps, one RHS: a kz plane (z-first) or a kx column plane (x-first)
  const size_t per_plane = xpipe ? (size_t)3 * g.My * g.nz : (size_t)3 * g.ny * g.Mx;
  const int nplanes_all = xpipe ? g.Mx : g.Mz;
  if (nrhs <= zcap && zhat) return 0;
  if (zhat) { cudaFree(zhat); bytes_allocated -= (size_t)zcap * per_rhs_z * sizeof(C); zhat = nullptr; }
  if (slab) { cudaFree(slab); bytes_allocated -= (size_t)slab_nr * slab_B * per_plane * sizeof(C); slab = nullptr; }
  zcap = nrhs;
  cudaError_t e = cudaMalloc((void**)&zhat, (size_t)zcap * per_rhs_z * sizeof(C));
  if (e != cudaSuccess) { zcap = 0; set_cuda_error("malloc z-spectrum workspace", e); return 1; }
  bytes_allocated += (size_t)zcap * per_rhs_z * sizeof(C);
  if (slices_layout) {
    // bounded memory: the middle stage holds max(4, planes/16) planes of one
    // RHS, and at least 32 MiB of them, so that its launches fill the GPU on
    // small grids (128^3: 6 batches of 43 planes instead of 16 of 16); the
    // batches are balanced
    slab_nr = 1;
    const size_t floor_planes = ceil_div((size_t)32 << 20, per_plane * sizeof(C));
    const int want = (int)std::max<size_t>({(size_t)4, (size_t)nplanes_all / 16, floor_planes});
    slab_B = std::min(nplanes_all, want);
    slab_B = (int)ceil_div((size_t)nplanes_all, ceil_div((size_t)nplanes_all, (size_t)slab_B));
  } else {
    const size_t full_rhs = per_plane * nplanes_all;
    if (full_rhs * zcap <= slab_budget_elems) { slab_nr = zcap; slab_B = nplanes_all; }
    else if (full_rhs <= slab_budget_elems) { slab_nr = (int)std::max<size_t>(1, slab_budget_elems / full_rhs); slab_B = nplanes_all; }
    else { slab_nr = 1; slab_B = (int)std::max<size_t>(1, slab_budget_elems / per_plane); }
  }
  e = cudaMalloc((void**)&slab, (size_t)slab_nr * slab_B * per_plane * sizeof(C));
  if (e != cudaSuccess) { set_cuda_error("malloc xy-slab workspace", e); return 1; }
  bytes_allocated += (size_t)slab_nr * slab_B * per_plane * sizeof(C);
  return 0;
}


template <typename T> int Engine<T>::matvec(const MvArgs<T>& a) {
  raise_smem_limit((const void*)k_zfwd<T>);
  raise_smem_limit((const void*)k_xfwd<T>);
  raise_smem_limit((const void*)k_ygreen<T>);
  raise_smem_limit((const void*)k_xinv<T>);
  raise_smem_limit((const void*)k_zinv_fin<T>);
  {
    // z-spectrum capacity: all RHS of the call if they fit the budget
    const size_t per_rhs_z = zhat_per_rhs() * sizeof(C);
    const size_t budget = (size_t)env_int("DDSCAT_B200_ZHAT_MB", 16384) * 1024 * 1024;
    const int want = (int)std::max<size_t>(1, std::min<size_t>((size_t)a.nrhs, budget / per_rhs_z));
    if (ensure_workspace(want)) return 1;
  }
  if (xpipe) return matvec_xpipe<T>(*this, a);
  MvParams<T> P{};
  P.nx = g.nx; P.ny = g.ny; P.nz = g.nz; P.Mx = g.Mx; P.My = g.My; P.Mz = g.Mz;
  P.nat = g.nat; P.nat0 = g.nat0;
  P.x_rs = a.x_rs; P.y_rs = a.y_rs; P.a_rs = a.a_rs;
  P.io_full = a.io_full; P.a_full = a.a_full; P.conj = a.conj;
  P.inv = inv; P.iocc = iocc; P.mask = a.mask;
  P.zhat = zhat; P.zhat_rs = (size_t)3 * g.Mz * g.ny * g.nx;
  P.slab = slab;
  P.green = green; P.ipbc = g.ipbc;
  P.px = px; P.py = py; P.pz = pz;
  P.twx = twx; P.twy = twy; P.twz = twz;
  P.inv_ngrid = (T)(1.0 / (double)g.ngrid());
  const int tile_elems = tune_tile > 0 ? tune_tile : ((sizeof(C) == 8) ? 4096 : 2048);  // 32 KiB by default
  P.tz = std::max(1, std::min(32, tile_elems / g.Mz));
  P.ry = std::max(1, std::min(16, tile_elems / (g.Mx + 1)));
  P.ty = std::max(1, std::min(32, (tile_elems / 2) / g.My));
  const int threads = 256;
  // per-pass kernel, grid geometry and shared memory: register path or generic
  const void* fz_r = pick_reg<T>(Pass::ZF, g.Mz);
  const void* fx_r = pick_reg<T>(Pass::XF, g.Mx);
  const void* fy_r = pick_reg<T>(Pass::YG, g.My);
  const void* fxi_r = pick_reg<T>(Pass::XI, g.Mx);
  const void* fzi_r = pick_reg<T>(Pass::ZI, g.Mz);
  // block sizes of the register passes (threads): z columns, x rows, y columns
  const int thz = tune_thz, thx = tune_thx;
  const int Ly = tune_ly;  // y-pass columns per block
  const int thy = 3 * reg_T(g.My) * Ly;
  const int Lz = thz / reg_T(g.Mz), Rx = thx / reg_T(g.Mx);
  P.lsz = line_stride(reg_E(g.Mz), reg_T(g.Mz), Lz, true);
  P.lsx = line_stride(reg_E(g.Mx), reg_T(g.Mx), Rx, false);
  P.lsy = std::max(line_stride(reg_E(g.My), reg_T(g.My), Ly, true), g.My);
  const size_t smz_r = ((size_t)Lz * P.lsz + g.Mz) * sizeof(C);
  const size_t smx_r = ((size_t)Rx * P.lsx + g.Mx) * sizeof(C);
  const size_t smy_r = ((size_t)3 * Ly * P.lsy + g.My) * sizeof(C);
  const size_t sm_z = (size_t)2 * P.tz * g.Mz * sizeof(C);
  const size_t sm_x = (size_t)2 * P.ry * (g.Mx + 1) * sizeof(C);
  const size_t sm_y = (size_t)4 * P.ty * g.My * sizeof(C);
  for (const void* f : {fz_r, fx_r, fy_r, fxi_r, fzi_r})
    if (f) raise_smem_limit(f);
  for (int r0 = 0; r0 < a.nrhs; r0 += zcap) {
    const int nr = std::min(zcap, a.nrhs - r0);
    P.rhs0 = r0;
    P.x = a.x + (size_t)r0 * a.x_rs;
    P.y = a.y + (size_t)r0 * a.y_rs;
    P.adia = a.adia + (size_t)r0 * a.a_rs;
    P.aoff = a.aoff ? a.aoff + (size_t)r0 * a.a_rs : nullptr;
    if (fz_r) {
      if (launch_k<T>(fz_r, dim3((unsigned)ceil_div(g.nx, Lz), (unsigned)g.ny, (unsigned)(3 * nr)), thz, smz_r, stream, P)) return 21;
    } else {
      dim3 gz((unsigned)ceil_div(g.nx, P.tz), (unsigned)g.ny, (unsigned)(3 * nr));
      k_zfwd<T><<<gz, threads, sm_z, stream>>>(P);
      note_launch();
      if (check_launch("MATVEC z-forward")) return 21;
    }
    for (int rs = 0; rs < nr; rs += slab_nr) {
      const int nrs = std::min(slab_nr, nr - rs);
      P.slab_rhs0 = rs;
      for (int kz0 = 0; kz0 < g.Mz; kz0 += slab_B) {
        P.kz0 = kz0;
        P.nplanes = std::min(slab_B, g.Mz - kz0);
        if (fx_r) {
          if (launch_k<T>(fx_r, dim3((unsigned)ceil_div(g.ny, Rx), (unsigned)P.nplanes, (unsigned)(3 * nrs)), thx, smx_r, stream, P)) return 22;
        } else {
          dim3 gx((unsigned)ceil_div(g.ny, P.ry), (unsigned)P.nplanes, (unsigned)(3 * nrs));
          k_xfwd<T><<<gx, threads, sm_x, stream>>>(P);
          note_launch();
          if (check_launch("MATVEC x-forward")) return 22;
        }
        if (fy_r) {
          if (launch_k<T>(fy_r, dim3((unsigned)nrs, (unsigned)ceil_div(g.Mx, Ly), (unsigned)P.nplanes), thy, smy_r, stream, P)) return 23;
        } else {
          dim3 gy((unsigned)ceil_div(g.Mx, P.ty), (unsigned)P.nplanes, (unsigned)nrs);
          k_ygreen<T><<<gy, threads, sm_y, stream>>>(P);
          note_launch();
          if (check_launch("MATVEC y-Green")) return 23;
        }
        if (fxi_r) {
          if (launch_k<T>(fxi_r, dim3((unsigned)ceil_div(g.ny, Rx), (unsigned)P.nplanes, (unsigned)(3 * nrs)), thx, smx_r, stream, P)) return 24;
        } else {
          dim3 gx((unsigned)ceil_div(g.ny, P.ry), (unsigned)P.nplanes, (unsigned)(3 * nrs));
          k_xinv<T><<<gx, threads, sm_x, stream>>>(P);
          note_launch();
          if (check_launch("MATVEC x-inverse")) return 24;
        }
      }
    }
    if (fzi_r) {
      if (launch_k<T>(fzi_r, dim3((unsigned)ceil_div(g.nx, Lz), (unsigned)g.ny, (unsigned)(3 * nr)), thz, smz_r, stream, P)) return 25;
    } else {
      dim3 gz((unsigned)ceil_div(g.nx, P.tz), (unsigned)g.ny, (unsigned)(3 * nr));
      k_zinv_fin<T><<<gz, threads, sm_z, stream>>>(P);
      note_launch();
      if (check_launch("MATVEC z-inverse/finish")) return 25;
    }
  }
  return 0;
}

template <typename C> __global__ void k_interleave6(const C* src, C* dst, size_t npts) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 6 * npts; i += (size_t)gridDim.x * blockDim.x) {
    const size_t m = i / npts, p = i - m * npts;
    dst[p * 6 + m] = src[i];
  }
}

// planar [6][points] (CXZC / build layout) -> point-interleaved [points][6] in `green`
template <typename T> int Engine<T>::interleave_green(const C* planar_dev) {
  if (xpipe) return interleave_green_zfast<T>(*this, planar_dev);
  const size_t npts = g.green_count() / 6;
  k_interleave6<C><<<(unsigned)std::min<size_t>(ceil_div(6 * npts, 256), 148 * 32), 256, 0, stream>>>(planar_dev, green, npts);
  note_launch();
  return check_launch("Green interleave");
}

template <typename T> int Engine<T>::upload_green(const void* host_green) {
  C* tmp = nullptr;
  cudaError_t e = cudaMalloc((void**)&tmp, g.green_count() * sizeof(C));
  if (e == cudaSuccess) e = cudaMemcpy(tmp, host_green, g.green_count() * sizeof(C), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(tmp); set_cuda_error("green H2D", e); return 4; }
  int rc = interleave_green(tmp);
  e = cudaStreamSynchronize(stream);
  cudaFree(tmp);
  if (rc || e != cudaSuccess) { if (!rc) set_cuda_error("green interleave", e); return 4; }
  return 0;
}

template <typename T> void Engine<T>::release() {
  cudaFree(twx); cudaFree(twy); cudaFree(twz);
  cudaFree(green); cudaFree(occ); cudaFree(inv); cudaFree(iocc); cudaFree(rowq);
  cudaFree(zhat); cudaFree(slab); cudaFree(d_err);
  *this = Engine<T>{};
}

// ---------------------------------------------------------------- autotuner
// Candidate launch shapes are those that change a kernel this grid uses:
// power-of-two axes run register passes (block sizes, y columns per block),
// the other axes run generic Stockham passes (tile size).  Each candidate is
// timed with CUDA events over `iters` single-RHS MATVECs after two warm-up
// calls; the x-first pipeline has no launch-shape choices and is left alone.
int autotune_engine(Engine<float>& e, int iters, float* default_ms, float* best_ms) {
  using C = float2;
  const Geometry& g = e.g;
  const size_t cn = (size_t)3 * g.nat0;
  C *x = nullptr, *y = nullptr, *ad = nullptr;
  cudaError_t err = cudaMalloc((void**)&x, cn * sizeof(C));
  if (err == cudaSuccess) err = cudaMalloc((void**)&y, cn * sizeof(C));
  if (err == cudaSuccess) err = cudaMalloc((void**)&ad, cn * sizeof(C));
  if (err != cudaSuccess) { cudaFree(x); cudaFree(y); cudaFree(ad); set_cuda_error("autotune", err); return 1; }
  cudaMemsetAsync(x, 0, cn * sizeof(C), e.stream);
  cudaMemsetAsync(ad, 0, cn * sizeof(C), e.stream);
  MvArgs<float> a;
  a.x = x; a.x_rs = cn; a.y = y; a.y_rs = cn; a.io_full = 0;
  a.adia = ad; a.a_rs = cn; a.a_full = 0; a.aoff = nullptr; a.conj = 0; a.nrhs = 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto time_it = [&](float* ms) -> int {
    for (int w = 0; w < 2; ++w)
      if (e.matvec(a)) return 1;
    cudaEventRecord(e0, e.stream);
    for (int i = 0; i < iters; ++i)
      if (e.matvec(a)) return 1;
    cudaEventRecord(e1, e.stream);
    if (cudaEventSynchronize(e1) != cudaSuccess) return 1;
    cudaEventElapsedTime(ms, e0, e1);
    *ms /= iters;
    return 0;
  };
  struct Shape { int thz, thx, ly, tile, zg; };
  const Shape def{e.tune_thz, e.tune_thx, e.tune_ly, e.tune_tile, e.tune_zg};
  std::vector<Shape> cands{def};
  if (e.xpipe) {
    // the two z passes of the x-first pipeline, where both apply (E <= 16)
    if (xzg3_supported(g.Mz)) cands.push_back({def.thz, def.thx, def.ly, def.tile, 1 - def.zg});
  } else {
    const bool rz = reg_supported(g.Mz), rx = reg_supported(g.Mx), ry = reg_supported(g.My);
    const std::vector<int> thzs = rz ? std::vector<int>{128, 256} : std::vector<int>{def.thz};
    const std::vector<int> thxs = rx ? std::vector<int>{128, 256} : std::vector<int>{def.thx};
    std::vector<int> lys{def.ly};
    if (ry)
      for (int ly : {1, 2, 4, 8})
        if (3 * reg_T(g.My) * ly <= 384) lys.push_back(ly);
    std::vector<int> tiles{def.tile};
    if (!(rz && rx && ry)) tiles = {0, 1024, 4096};
    for (int a1 : thzs)
      for (int a2 : thxs)
        for (int a3 : lys)
          for (int a4 : tiles) cands.push_back({a1, a2, a3, a4, def.zg});
  }
  int rc = 0;
  float dms = 0.f, bms = 0.f;
  Shape best = def;
  for (size_t k = 0; k < cands.size() && !rc; ++k) {
    e.tune_thz = cands[k].thz; e.tune_thx = cands[k].thx; e.tune_ly = cands[k].ly; e.tune_tile = cands[k].tile;
    e.tune_zg = cands[k].zg;
    float ms = 0.f;
    if (time_it(&ms)) {
      if (k == 0) { rc = 1; break; }  // the default shape must run
      cudaGetLastError();             // a rejected candidate (launch limits) is skipped
      continue;
    }
    if (k == 0) { dms = bms = ms; continue; }
    if (ms < bms) { bms = ms; best = cands[k]; }
  }
  e.tune_thz = best.thz; e.tune_thx = best.thx; e.tune_ly = best.ly; e.tune_tile = best.tile;
  e.tune_zg = best.zg;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(x); cudaFree(y); cudaFree(ad);
  if (rc) return 1;
  *default_ms = dms;
  *best_ms = bms;
  clear_error();
  return 0;
}

template struct Engine<float>;
template struct Engine<double>;

}  // namespace ddb
