// Batched multi-RHS Krylov solves (sm_100a): masked per-RHS vector kernels,
// per-RHS FP64 inner products in one launch, and the QMRCCG / PBCGS2
// recurrences of solvers.cu run for every RHS in lock-step.  Host syncs (one
// small D2H per group of inner products) are shared by all RHS of the batch.
#include <algorithm>
#include <complex>
#include <condition_variable>
#include <mutex>
#include "batch.h"
#include <cstdio>
#include <cstdlib>

namespace ddb {

using Z = std::complex<double>;
static inline double2 dz(Z z) { return make_double2(z.real(), z.imag()); }
static inline Z zd2(double2 v) { return Z(v.x, v.y); }

constexpr int BT = 256;

template <typename C>
__global__ void __launch_bounds__(BT) kb_lin(int n, C* d, const double2* cd, const C* a, const double2* ca, const C* b,
                                             const double2* cb, const int* mask) {
  const int r = blockIdx.y;
  if (mask && !mask[r]) return;
  const size_t off = (size_t)r * n;
  const double2 zd = cd ? cd[r] : make_double2(0.0, 0.0);
  const double2 za = ca ? ca[r] : make_double2(0.0, 0.0);
  const double2 zb = cb ? cb[r] : make_double2(0.0, 0.0);
  const bool keep = cd && !(zd.x == 0.0 && zd.y == 0.0);
  const bool d1 = zd.x == 1.0 && zd.y == 0.0, a1 = za.x == 1.0 && za.y == 0.0, b1 = zb.x == 1.0 && zb.y == 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    C v = mk<C>(0, 0);
    if (keep) v = d1 ? d[off + i] : zmulv(zd, d[off + i]);
    if (a) v = cadd(v, a1 ? a[off + i] : zmulv(za, a[off + i]));
    if (b) v = cadd(v, b1 ? b[off + i] : zmulv(zb, b[off + i]));
    d[off + i] = v;
  }
}

template <typename T> struct BDot {
  const cplx<T>* a[8];
  const cplx<T>* b[8];
  const cplx<T>* c[8];
  int conj[8];
  int K, mode;  // mode 0: products; 1: (|a-b|^2, |a-b-c|^2)
};

__device__ __forceinline__ double2 wsum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}

template <typename T>
__global__ void __launch_bounds__(BT) kb_dots(int n, BDot<T> sp, const int* mask, double2* part, double2* out,
                                              unsigned* cnt) {
  __shared__ double2 ws[8][BT / 32];
  __shared__ bool last;
  const int r = blockIdx.y;
  if (mask && !mask[r]) return;
  const size_t off = (size_t)r * n;
  double2 acc[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) acc[k] = make_double2(0.0, 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (sp.mode == 0) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (k >= sp.K) break;
        const double2 a = to_d(sp.a[k][off + i]), b = to_d(sp.b[k][off + i]);
        if (sp.conj[k]) { acc[k].x += a.x * b.x + a.y * b.y; acc[k].y += a.x * b.y - a.y * b.x; }
        else { acc[k].x += a.x * b.x - a.y * b.y; acc[k].y += a.x * b.y + a.y * b.x; }
      }
    } else {
      const double2 a = to_d(sp.a[0][off + i]), b = to_d(sp.b[0][off + i]), c = to_d(sp.c[0][off + i]);
      const double dr = a.x - b.x, di = a.y - b.y;
      acc[0].x += dr * dr + di * di;
      const double er = dr - c.x, ei = di - c.y;
      acc[1].x += er * er + ei * ei;
    }
  }
  // the loops over k stay unrolled with compile-time indices so that acc
  // lives in registers
  const int K = sp.mode == 0 ? sp.K : 2;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (k >= K) break;
    const double2 v = wsum2(acc[k]);
    if (lane == 0) ws[k][wid] = v;
  }
  __syncthreads();
  double2* P = part + ((size_t)r * 8) * gridDim.x;
  if (threadIdx.x < 32) {
    for (int k = 0; k < K; ++k) {
      double2 v = lane < BT / 32 ? ws[k][lane] : make_double2(0.0, 0.0);
      v = wsum2(v);
      if (lane == 0) P[(size_t)k * gridDim.x + blockIdx.x] = v;
    }
  }
  __threadfence();
  if (threadIdx.x == 0) last = atomicInc(cnt + r, gridDim.x - 1) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = 0; k < K; ++k) {
    double2 v = make_double2(0.0, 0.0);
    for (int bi = threadIdx.x; bi < (int)gridDim.x; bi += blockDim.x) {
      const volatile double* pp = reinterpret_cast<volatile double*>(P + (size_t)k * gridDim.x + bi);
      v.x += pp[0];
      v.y += pp[1];
    }
    v = wsum2(v);
    if (lane == 0) ws[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int k = 0; k < K; ++k) {
      double2 v = lane < BT / 32 ? ws[k][lane] : make_double2(0.0, 0.0);
      v = wsum2(v);
      if (lane == 0) out[(size_t)r * 8 + k] = v;
    }
  }
}

// Block partial sums of NK (<= 2) FP64 accumulators into part[r][k0 + k][block],
// and the last block of RHS r (in completion order) folds all partials in a
// fixed order into out[r][k0 + k]: deterministic for a given grid.
template <int NK>
__device__ __forceinline__ void block_sums(const double2 (&acc)[NK], int k0, int r, double2* part, double2* out,
                                           unsigned* cnt) {
  __shared__ double2 ws[NK][BT / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    const double2 v = wsum2(acc[k]);
    if (lane == 0) ws[k][wid] = v;
  }
  __syncthreads();
  double2* P = part + ((size_t)r * 8) * gridDim.x;
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double2 v = lane < BT / 32 ? ws[k][lane] : make_double2(0.0, 0.0);
      v = wsum2(v);
      if (lane == 0) P[(size_t)(k0 + k) * gridDim.x + blockIdx.x] = v;
    }
  }
  __threadfence();
  if (threadIdx.x == 0) last = atomicInc(cnt + r, gridDim.x - 1) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NK; ++k) {
    double2 v = make_double2(0.0, 0.0);
    for (int bi = threadIdx.x; bi < (int)gridDim.x; bi += blockDim.x) {
      const volatile double* pp = reinterpret_cast<volatile double*>(P + (size_t)(k0 + k) * gridDim.x + bi);
      v.x += pp[0];
      v.y += pp[1];
    }
    v = wsum2(v);
    __syncthreads();
    if (lane == 0) ws[k][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
#pragma unroll
    for (int k = 0; k < NK; ++k) {
      double2 v = lane < BT / 32 ? ws[k][lane] : make_double2(0.0, 0.0);
      v = wsum2(v);
      if (lane == 0) out[(size_t)r * 8 + k0 + k] = v;
    }
  }
}

// One-MATVEC QMRCCG, first vector step of an iteration, per RHS r in mask:
//   p = cp p + cv vt ; q = cq q + cw atw ; vt = ct vt + q
// with sums |vt|^2 and vt^T vt into out slots k0, k0+1.  Same element
// arithmetic as the separate kb_lin updates it replaces.
template <typename C>
__global__ void __launch_bounds__(BT) kq_pqv(int n, C* p, C* q, C* vt, const C* atw, const double2* co,
                                             const int* mask, int k0, double2* part, double2* out, unsigned* cnt) {
  const int r = blockIdx.y, R = gridDim.y;
  if (mask && !mask[r]) return;
  const size_t off = (size_t)r * n;
  const double2 cp = co[r], cv = co[R + r], cq = co[2 * R + r], cw = co[3 * R + r], ct = co[4 * R + r];
  double2 acc[2] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
  for (int i = blockIdx.x * BT + threadIdx.x; i < n; i += gridDim.x * BT) {
    const C v0 = vt[off + i];
    const C pn = cadd(zmulv(cp, p[off + i]), zmulv(cv, v0));
    const C qn = cadd(zmulv(cq, q[off + i]), zmulv(cw, atw[off + i]));
    const C vn = cadd(zmulv(ct, v0), qn);
    p[off + i] = pn;
    q[off + i] = qn;
    vt[off + i] = vn;
    const double2 a = to_d(vn);
    acc[0].x += a.x * a.x + a.y * a.y;
    acc[1].x += a.x * a.x - a.y * a.y;
    acc[1].y += 2.0 * a.x * a.y;
  }
  block_sums<2>(acc, k0, r, part, out, cnt);
}

// One-MATVEC QMRCCG, last vector step of an iteration, per RHS r in mask:
//   d = th d + ka p ; s = th s + ka q ; x = x + d ; r = r - s
// with the sum |r|^2 into out slot k0.
template <typename C>
__global__ void __launch_bounds__(BT) kq_dsxr(int n, C* d, C* s, C* x, C* rv, const C* p, const C* q,
                                              const double2* co, const int* mask, int k0, double2* part,
                                              double2* out, unsigned* cnt) {
  const int r = blockIdx.y, R = gridDim.y;
  if (mask && !mask[r]) return;
  const size_t off = (size_t)r * n;
  const double2 th = co[r], ka = co[R + r];
  double2 acc[1] = {make_double2(0.0, 0.0)};
  for (int i = blockIdx.x * BT + threadIdx.x; i < n; i += gridDim.x * BT) {
    const C dn = cadd(zmulv(th, d[off + i]), zmulv(ka, p[off + i]));
    const C sn = cadd(zmulv(th, s[off + i]), zmulv(ka, q[off + i]));
    const C xn = cadd(x[off + i], dn);
    const C rn = csub(rv[off + i], sn);
    d[off + i] = dn;
    s[off + i] = sn;
    x[off + i] = xn;
    rv[off + i] = rn;
    const double2 a = to_d(rn);
    acc[0].x += a.x * a.x + a.y * a.y;
  }
  block_sums<1>(acc, k0, r, part, out, cnt);
}

// One-MATVEC QMRCCG, the last vector step of iteration k fused with the first
// of iteration k+1 (they read the same p and q), per RHS r in mask:
//   d = th d + ka p ; s = th s + ka q ; x = x + d ; r = r - s          (k)
//   p = cp p + cv vt ; q = cq q + cw atw ; vt = ct vt + q              (k+1)
// with |r|^2 into out slot 0, |vt|^2 and vt^T vt into slots 2 and 3 (slot 1
// is written 0).  co holds the five k+1 coefficients, then th and ka.  Same
// element arithmetic and reduction grid as kq_dsxr and kq_pqv.
template <typename C>
__global__ void __launch_bounds__(BT) kq_dsxr_pqv(int n, C* __restrict__ d, C* __restrict__ s, C* __restrict__ x,
                                                  C* __restrict__ rv, C* __restrict__ p, C* __restrict__ q,
                                                  C* __restrict__ vt, const C* __restrict__ atw, const double2* co,
                                                  const int* mask, double2* part, double2* out, unsigned* cnt) {
  const int r = blockIdx.y, R = gridDim.y;
  if (mask && !mask[r]) return;
  const size_t off = (size_t)r * n;
  d += off; s += off; x += off; rv += off; p += off; q += off; vt += off; atw += off;
  const double2 cp = co[r], cv = co[R + r], cq = co[2 * R + r], cw = co[3 * R + r], ct = co[4 * R + r];
  const double2 th = co[5 * R + r], ka = co[6 * R + r];
  double2 acc[4] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
  // two elements per thread and round: all sixteen loads are issued before the stores
  const int stride = gridDim.x * BT;
  for (int i0 = blockIdx.x * BT + threadIdx.x; i0 < n; i0 += 2 * stride) {
    C p0[2], q0[2], v0[2], a0[2], d0[2], s0[2], x0[2], r0[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = i0 + k * stride;
      if (i < n) {
        p0[k] = p[i]; q0[k] = q[i]; v0[k] = vt[i]; a0[k] = atw[i];
        d0[k] = d[i]; s0[k] = s[i]; x0[k] = x[i]; r0[k] = rv[i];
      }
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = i0 + k * stride;
      if (i >= n) break;
      const C dn = cadd(zmulv(th, d0[k]), zmulv(ka, p0[k]));
      const C sn = cadd(zmulv(th, s0[k]), zmulv(ka, q0[k]));
      const C xn = cadd(x0[k], dn);
      const C rn = csub(r0[k], sn);
      const C pn = cadd(zmulv(cp, p0[k]), zmulv(cv, v0[k]));
      const C qn = cadd(zmulv(cq, q0[k]), zmulv(cw, a0[k]));
      const C vn = cadd(zmulv(ct, v0[k]), qn);
      d[i] = dn;
      s[i] = sn;
      x[i] = xn;
      rv[i] = rn;
      p[i] = pn;
      q[i] = qn;
      vt[i] = vn;
      const double2 a = to_d(rn), b = to_d(vn);
      acc[0].x += a.x * a.x + a.y * a.y;
      acc[2].x += b.x * b.x + b.y * b.y;
      acc[3].x += b.x * b.x - b.y * b.y;
      acc[3].y += 2.0 * b.x * b.y;
    }
  }
  block_sums<4>(acc, 0, r, part, out, cnt);
}

template <typename T> int BatchOps<T>::init(int R_, int n_, cudaStream_t s) {
  R = R_;
  n = n_;
  stream = s;
  nb = (int)std::max<size_t>(1, std::min<size_t>(ceil_div(n, BT), std::max(1, 592 / std::max(1, R))));
  coef_cap = (size_t)3 * R * 96;
  cudaError_t e = cudaMalloc((void**)&d_part, (size_t)R * 8 * nb * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_out, (size_t)R * 8 * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_cnt, (size_t)R * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h_out, (size_t)R * 8 * sizeof(double2));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h_coef, coef_cap * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_coef, coef_cap * sizeof(double2));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h_mask, (size_t)MASKS * R * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_masks, (size_t)MASKS * R * sizeof(int));
  if (e != cudaSuccess) { set_cuda_error("batch buffers", e); return 1; }
  cudaMemset(d_cnt, 0, (size_t)R * sizeof(unsigned));
  return 0;
}

template <typename T> void BatchOps<T>::release() {
  cudaFree(d_part); cudaFree(d_out); cudaFree(d_cnt); cudaFree(d_coef); cudaFree(d_masks);
  if (h_out) cudaFreeHost(h_out);
  if (h_coef) cudaFreeHost(h_coef);
  if (h_mask) cudaFreeHost(h_mask);
  *this = BatchOps<T>{};
}

template <typename T> const int* BatchOps<T>::mask(const std::vector<int>& m) {
  if (mask_pos >= (size_t)MASKS) {  // ring full: wait for pending copies, then reuse
    cudaStreamSynchronize(stream);
    mask_pos = 0;
  }
  int* h = h_mask + mask_pos * R;
  int* d = d_masks + mask_pos * R;
  for (int r = 0; r < R; ++r) h[r] = m[r];
  cudaMemcpyAsync(d, h, (size_t)R * sizeof(int), cudaMemcpyHostToDevice, stream);
  ++mask_pos;
  return d;
}

template <typename T>
int BatchOps<T>::lin(C* d, const double2* zd, const C* a, const double2* za, const C* b, const double2* zb,
                     const int* msk) {
  if (coef_pos + 3 * (size_t)R > coef_cap) {
    cudaStreamSynchronize(stream);
    coef_pos = 0;
  }
  double2* h = h_coef + coef_pos;
  double2* dc = d_coef + coef_pos;
  const double2* src[3] = {zd, za, zb};
  for (int k = 0; k < 3; ++k)
    for (int r = 0; r < R; ++r) h[k * R + r] = src[k] ? src[k][r] : make_double2(0.0, 0.0);
  cudaMemcpyAsync(dc, h, (size_t)3 * R * sizeof(double2), cudaMemcpyHostToDevice, stream);
  coef_pos += 3 * (size_t)R;
  const unsigned gx = (unsigned)std::max<size_t>(1, std::min<size_t>(ceil_div(n, BT), std::max(1, 2368 / R)));
  kb_lin<C><<<dim3(gx, R), BT, 0, stream>>>(n, d, zd ? dc : nullptr, a, za ? dc + R : nullptr, b, zb ? dc + 2 * R : nullptr,
                                            msk);
  note_launch();
  return check_launch("batched vector update");
}

template <typename T> const double2* BatchOps<T>::upload(const std::vector<const double2*>& cols) {
  const size_t need = cols.size() * (size_t)R;
  if (coef_pos + need > coef_cap) {
    cudaStreamSynchronize(stream);
    coef_pos = 0;
  }
  double2* h = h_coef + coef_pos;
  double2* dc = d_coef + coef_pos;
  for (size_t k = 0; k < cols.size(); ++k)
    for (int r = 0; r < R; ++r) h[k * R + r] = cols[k][r];
  cudaMemcpyAsync(dc, h, need * sizeof(double2), cudaMemcpyHostToDevice, stream);
  coef_pos += need;
  return dc;
}

template <typename T>
int BatchOps<T>::qmr_pqv(C* p, C* q, C* vt, const C* atw, const double2* cp, const double2* cv, const double2* cq,
                         const double2* cw, const double2* ct, const int* msk) {
  const double2* co = upload({cp, cv, cq, cw, ct});
  kq_pqv<C><<<dim3(nb, R), BT, 0, stream>>>(n, p, q, vt, atw, co, msk, 2, d_part, d_out, d_cnt);
  note_launch();
  return check_launch("batched QMR p/q/v update");
}

template <typename T>
int BatchOps<T>::qmr_dsxr(C* d, C* s, C* x, C* r, const C* p, const C* q, const double2* th, const double2* ka,
                          const int* msk, std::vector<double2>& rr) {
  const double2* co = upload({th, ka});
  kq_dsxr<C><<<dim3(nb, R), BT, 0, stream>>>(n, d, s, x, r, p, q, co, msk, 0, d_part, d_out, d_cnt);
  note_launch();
  if (check_launch("batched QMR d/s/x/r update")) return 1;
  cudaError_t e = cudaMemcpyAsync(h_out, d_out, (size_t)R * 8 * sizeof(double2), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) { set_cuda_error("batched QMR update D2H", e); return 1; }
  reset_ring();
  rr.assign((size_t)R, make_double2(0, 0));
  for (int i = 0; i < R; ++i) rr[i] = h_out[(size_t)i * 8];
  return 0;
}

template <typename T> int BatchOps<T>::copy(C* d, const C* a, const int* msk) {
  std::vector<double2> one(R, make_double2(1.0, 0.0));
  return lin(d, nullptr, a, one.data(), nullptr, nullptr, msk);
}

template <typename T> int BatchOps<T>::zero(C* d, const int* msk) {
  return lin(d, nullptr, nullptr, nullptr, nullptr, nullptr, msk);
}

template <typename T>
int BatchOps<T>::dots(int K, const C* const* a, const C* const* b, const int* conj, const int* msk,
                      std::vector<double2>& out) {
  BDot<T> sp{};
  sp.K = K;
  sp.mode = 0;
  for (int k = 0; k < K; ++k) { sp.a[k] = a[k]; sp.b[k] = b[k]; sp.conj[k] = conj[k]; }
  kb_dots<T><<<dim3(nb, R), BT, 0, stream>>>(n, sp, msk, d_part, d_out, d_cnt);
  note_launch();
  if (check_launch("batched inner products")) return 1;
  cudaError_t e = cudaMemcpyAsync(h_out, d_out, (size_t)R * 8 * sizeof(double2), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) { set_cuda_error("batched inner products D2H", e); return 1; }
  reset_ring();
  out.assign((size_t)R * K, make_double2(0, 0));
  for (int r = 0; r < R; ++r)
    for (int k = 0; k < K; ++k) out[(size_t)r * K + k] = h_out[(size_t)r * 8 + k];
  return 0;
}

template <typename T>
int BatchOps<T>::diff_norms(const C* a, const C* b, const C* c, const int* msk, std::vector<double2>& out) {
  BDot<T> sp{};
  sp.K = 2;
  sp.mode = 1;
  sp.a[0] = a; sp.b[0] = b; sp.c[0] = c;
  kb_dots<T><<<dim3(nb, R), BT, 0, stream>>>(n, sp, msk, d_part, d_out, d_cnt);
  note_launch();
  if (check_launch("batched residual norms")) return 1;
  cudaError_t e = cudaMemcpyAsync(h_out, d_out, (size_t)R * 8 * sizeof(double2), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) { set_cuda_error("batched residual norms D2H", e); return 1; }
  reset_ring();
  out.assign((size_t)R * 2, make_double2(0, 0));
  for (int r = 0; r < R; ++r) {
    out[(size_t)r * 2] = h_out[(size_t)r * 8];
    out[(size_t)r * 2 + 1] = h_out[(size_t)r * 8 + 1];
  }
  return 0;
}

// --------------------------------------------------------------------------
// shared solver plumbing
template <typename T> struct BCtx {
  using C = cplx<T>;
  BatchIO<T>& io;
  BatchOps<T>& ops;
  int R, n;
  std::vector<int> nc;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  int last_cnt = 0;  // RHS of the latest MATVEC (its events are ev.back())
  explicit BCtx(BatchIO<T>& s) : io(s), ops(*s.ops), R(s.R), n(s.n), nc(s.R, 0) {}
  ~BCtx() {
    for (auto& p : ev) { cudaEventDestroy(p.first); cudaEventDestroy(p.second); }
  }
  C* w(int slot) { return io.work + (size_t)slot * R * n; }
  // MATVEC of `in` into `out` for RHS in mask m (host copy hm for counting)
  int mv(const C* in, C* out, const std::vector<int>& hm) {
    int cnt = 0;
    for (int r = 0; r < R; ++r) cnt += hm[r] ? 1 : 0;
    if (!cnt) return 0;
    const int* dm = ops.mask(hm);
    MvArgs<T> a;
    a.x = in; a.x_rs = n; a.y = out; a.y_rs = n; a.io_full = 0;
    a.adia = io.adia; a.aoff = io.aoff; a.a_rs = n; a.a_full = 0;
    a.conj = 0; a.mask = dm; a.nrhs = R;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ops.stream);
    int rc = io.eng->matvec(a);
    cudaEventRecord(e1, ops.stream);
    ev.push_back({e0, e1});
    if (rc) return rc;
    for (int r = 0; r < R; ++r) nc[r] += hm[r] ? 1 : 0;
    last_cnt = cnt;
    io.matvec_rhs += cnt;
    io.matvec_calls += 1;
    return 0;
  }
  void finish_timing() {
    cudaStreamSynchronize(ops.stream);
    double ms = 0.0;
    for (auto& p : ev) {
      float t = 0.f;
      cudaEventElapsedTime(&t, p.first, p.second);
      ms += t;
    }
    io.matvec_ms += ms;
  }
  static std::vector<double2> vals(const std::vector<Z>& z) {
    std::vector<double2> o(z.size());
    for (size_t i = 0; i < z.size(); ++i) o[i] = dz(z[i]);
    return o;
  }
  static std::vector<double2> cst(int R, Z v) { return std::vector<double2>(R, dz(v)); }
};

static bool any_of(const std::vector<int>& m) {
  for (int v : m)
    if (v) return true;
  return false;
}

// --------------------------------------------------------------------------
// Device-driven one-MATVEC QMRCCG iteration (residual replacement), captured in
// a CUDA graph.  The per-RHS scalar recurrence, the masks and the reliable-
// residual bookkeeping run in single-thread kernels on FP64 state held on the
// GPU, so an iteration needs no host round trip; the reliable-residual check
// (a masked MATVEC, two norms and the replacement) sits in an IF conditional
// node that k_qg_post arms only when some RHS needs a check.  The host
// launches the graph repeatedly and reads the active-RHS count every few
// launches.  Arithmetic is that of the host-driven form (FP64 scalars).
struct QGState {
  double2 *gamma, *ksi, *rho, *eps, *mu, *tau, *lambda, *kappa, *theta;
  double2 *co;           // [7][R]: p/q/v coefficients (5), d/s coefficients (2)
  double2 *one, *mone;   // [R]
  double *bnorm, *resid;
  int *it, *live, *status, *nc, *I, *CK, *RP;
  int *active, *checks;  // [1] each
};

__device__ __forceinline__ double2 dmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a / b by Smith's scaled algorithm (R. L. Smith, CACM 5(8), 1962), which
// avoids the overflow and underflow of |b|^2 the way the host's complex
// division does, so a stagnating recurrence with extreme scalars takes the same
// breakdown decisions on the device as on the host
__device__ __forceinline__ double2 ddiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  const double r = b.x / b.y, d = b.y + b.x * r;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
__device__ __forceinline__ double2 dsc(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ bool dz0(double2 a) { return a.x == 0.0 && a.y == 0.0; }

// Phase stamps of the captured iteration (DDSCAT_B200_VERBOSE): the global
// timer at 7 points of iteration it, st[8*it + slot]; st[8*cap] counts the
// iterations (bounded by cap).
__global__ void k_qg_stamp(unsigned long long* st, int cap, int slot, int bump) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  unsigned long long* n = st + 8 * (size_t)cap;
  const unsigned long long it = *n;
  if (it < (unsigned long long)cap) st[8 * it + slot] = t;
  if (bump) *n = it + 1;
}

// coefficients of the p/q/v step of RHS r from gamma, ksi, mu, tau
__device__ __forceinline__ void qg_pqv_coefficients(int R, int r, const QGState& S) {
  const double2 g = S.gamma[r], k = S.ksi[r], mu = S.mu[r], t = S.tau[r];
  const double2 one = make_double2(1.0, 0.0);
  S.co[r] = dsc(-1.0, mu);                            // -mu
  S.co[R + r] = ddiv(one, g);                         // 1/gamma
  S.co[2 * R + r] = dsc(-1.0, ddiv(dmul(g, mu), k));  // -(gamma mu)/ksi
  S.co[3 * R + r] = ddiv(one, k);                     // 1/ksi
  S.co[4 * R + r] = dsc(-1.0, ddiv(t, g));            // -(tau/gamma)
}

// I = live and it < maxit and resid > tol; coefficients of the p/q/v step
__global__ void k_qg_begin(int R, int maxit, double tol, QGState S) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const int on = S.live[r] && S.it[r] < maxit && S.resid[r] > tol;
    S.I[r] = on;
    if (!on) continue;
    S.it[r] += 1;
    S.nc[r] += 1;
    qg_pqv_coefficients(R, r, S);
  }
}

// Start of the next iteration inside the captured body (its p/q/v step already
// ran in kq_dsxr_pqv): I, iteration and MATVEC counts, and the active count.
__global__ void k_qg_next(int R, int maxit, double tol, QGState S) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int r = 0; r < R; ++r) {
    const int on = S.live[r] && S.it[r] < maxit && S.resid[r] > tol;
    S.I[r] = on;
    if (on) { S.it[r] += 1; S.nc[r] += 1; }
    c += on;
  }
  *S.active = c;
}

// scalar recurrence from |vt|^2, vt^T vt (out slots 2, 3) and vt^T A vt (slot 0)
__global__ void k_qg_scalars(int R, QGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.I[r]) continue;
    const double2 gamma0 = S.gamma[r], ksi0 = S.ksi[r], rho0 = S.rho[r], tau0 = S.tau[r], kappa0 = S.kappa[r];
    const double g2 = out[(size_t)r * 8 + 2].x;
    const double2 gam = make_double2(sqrt(fmax(0.0, g2)), 0.0);
    const double2 ksi = gam;  // left Lanczos vectors equal the right ones
    const double2 rho = out[(size_t)r * 8 + 3], eps = out[(size_t)r * 8];
    S.gamma[r] = gam; S.ksi[r] = ksi; S.rho[r] = rho; S.eps[r] = eps;
    int st = 0;
    if (dz0(gam)) st = 6;
    const double2 den = dmul(dmul(gam, S.tau[r]), rho0);
    if (!st && dz0(den)) st = 12;
    double2 mu = S.mu[r];
    if (!st) { mu = ddiv(dmul(dmul(gamma0, ksi0), rho), den); if (dz0(rho)) st = 13; }
    double2 theta = S.theta[r], kappa = kappa0, lambda = S.lambda[r], tau = S.tau[r];
    if (!st) {
      const double2 gm = dmul(gam, mu);
      tau = ddiv(eps, rho);
      tau = make_double2(tau.x - gm.x, tau.y - gm.y);
      const double at0 = tau0.x * tau0.x + tau0.y * tau0.y, ag = gam.x * gam.x + gam.y * gam.y;
      const double2 den2 = make_double2(lambda.x * at0 + ag, lambda.y * at0);
      if (dz0(den2)) st = 14;
      else {
        theta = ddiv(make_double2((1.0 - lambda.x) * at0, -lambda.y * at0), den2);
        kappa = dsc(-1.0, ddiv(dmul(dmul(gamma0, make_double2(tau0.x, -tau0.y)), kappa0), den2));
        lambda = ddiv(make_double2(lambda.x * at0, lambda.y * at0), den2);
      }
    }
    S.mu[r] = mu; S.tau[r] = tau; S.theta[r] = theta; S.kappa[r] = kappa; S.lambda[r] = lambda;
    if (st) { S.status[r] = 58; S.live[r] = 0; S.I[r] = 0; }
    S.co[5 * R + r] = theta;
    S.co[6 * R + r] = kappa;
    if (!st) qg_pqv_coefficients(R, r, S);  // for the p/q/v step of the next iteration (kq_dsxr_pqv)
  }
}

// recursive residual, the check mask and the IF condition of the check body
__global__ void k_qg_post(int R, double tol, QGState S, const double2* out, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  int any = 0;
  for (int r = 0; r < R; ++r) {
    int ck = 0;
    if (S.I[r]) {
      S.resid[r] = sqrt(fmax(0.0, out[(size_t)r * 8].x)) / S.bnorm[r];
      ck = (S.it[r] % 20) == 0 || S.resid[r] <= tol;
      if (ck) S.nc[r] += 1;
    }
    S.CK[r] = ck;
    S.RP[r] = 0;
    any |= ck;
  }
  if (any) *S.checks += 1;
  cudaGraphSetConditional(h, any ? 1u : 0u);
}

// decisions of the reliable-residual check from |b - A x|^2, |b - A x - r|^2
__global__ void k_qg_check(int R, double tol, QGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.CK[r]) continue;
    const double tr = sqrt(fmax(0.0, out[(size_t)r * 8].x)), gapn = sqrt(fmax(0.0, out[(size_t)r * 8 + 1].x));
    const double tres = tr / S.bnorm[r];
    const double gap = tr > 0.0 ? gapn / tr : (gapn == 0.0 ? 0.0 : INFINITY);
    const bool conv = tres <= tol;
    const bool rest = gap >= 1.0e-3 || (S.resid[r] <= tol && !conv);
    if (conv) { S.resid[r] = tres; S.live[r] = 0; continue; }
    if (rest) { S.RP[r] = 1; S.resid[r] = tres; }
  }
}


// Runs the iterations of the one-MATVEC QMRCCG with residual replacement from
// the state the host-driven setup produced, until no RHS is active.
template <typename T>
static int qmr_graph_loop(BatchIO<T>& io, BatchOps<T>& ops, std::vector<int>& nc, cplx<T>* const* w,
                          cplx<T>* xs, std::vector<Z>* sc, std::vector<double>& bnorm, std::vector<double>& resid,
                          std::vector<int>& it, std::vector<int>& live, std::vector<int>& status,
                          double mv_ms_per_rhs) {
  using C = cplx<T>;
  const int R = io.R, n = io.n;
  C *r = w[0], *p = w[1], *q = w[3], *d = w[4], *s = w[5], *vt = w[6], *atw = w[8], *sy = w[9];
  // device state
  const size_t nz2 = (size_t)(9 + 7 + 2) * R, nd = (size_t)2 * R, ni = (size_t)7 * R + 2;
  unsigned char* blk = nullptr;
  cudaError_t e = cudaMalloc((void**)&blk, nz2 * sizeof(double2) + nd * sizeof(double) + ni * sizeof(int));
  if (e != cudaSuccess) { set_cuda_error("graph solve state", e); return 1; }
  QGState S;
  double2* z = reinterpret_cast<double2*>(blk);
  double2** zp[9] = {&S.gamma, &S.ksi, &S.rho, &S.eps, &S.mu, &S.tau, &S.lambda, &S.kappa, &S.theta};
  for (int k = 0; k < 9; ++k) *zp[k] = z + (size_t)k * R;
  S.co = z + (size_t)9 * R;
  S.one = z + (size_t)16 * R;
  S.mone = z + (size_t)17 * R;
  double* dd = reinterpret_cast<double*>(z + nz2);
  S.bnorm = dd; S.resid = dd + R;
  int* ii = reinterpret_cast<int*>(dd + nd);
  int** ip[7] = {&S.it, &S.live, &S.status, &S.nc, &S.I, &S.CK, &S.RP};
  for (int k = 0; k < 7; ++k) *ip[k] = ii + (size_t)k * R;
  S.active = ii + (size_t)7 * R;
  S.checks = S.active + 1;
  // initial device state (uploaded on the solve's own stream below)
  std::vector<double2> hz(nz2, make_double2(0, 0));
  for (int k = 0; k < 9; ++k)
    for (int i = 0; i < R; ++i) hz[(size_t)k * R + i] = dz(sc[k][i]);
  for (int i = 0; i < R; ++i) { hz[(size_t)16 * R + i] = make_double2(1, 0); hz[(size_t)17 * R + i] = make_double2(-1, 0); }
  std::vector<double> hd0(nd);
  for (int i = 0; i < R; ++i) { hd0[i] = bnorm[i]; hd0[R + i] = resid[i]; }
  std::vector<int> hi0(ni, 0);
  for (int i = 0; i < R; ++i) {
    hi0[i] = it[i]; hi0[R + i] = live[i]; hi0[2 * R + i] = status[i]; hi0[3 * R + i] = nc[i];
  }
  // phase stamps of the iterations (verbose only)
  const bool verbose = verbose_level() >= 2;
  const int scap = io.maxit + 64;
  unsigned long long* stamps = nullptr;
  if (verbose && cudaMalloc((void**)&stamps, (size_t)(8 * scap + 1) * sizeof(unsigned long long)) != cudaSuccess)
    stamps = nullptr;
  auto stamp = [&](cudaStream_t s_, int slot, int bump) {
    if (stamps) k_qg_stamp<<<1, 1, 0, s_>>>(stamps, scap, slot, bump);
  };
  // partials of the MATVEC-fused vt^T A vt (x-first pipeline); else a separate sum kernel
  double2* xpart = nullptr;
  if (io.eng->xpipe) {
    e = cudaMalloc((void**)&xpart, (size_t)R * xdot_blocks(io.eng->g) * sizeof(double2));
    if (e != cudaSuccess) { cudaFree(blk); cudaFree(stamps); set_cuda_error("graph solve state", e); return 1; }
  }
  cudaStream_t st = nullptr, st2 = nullptr;
  cudaStreamSynchronize(ops.stream);
  e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking);
  // Every upload is ordered on st: st does not synchronise with the legacy
  // default stream, so a plain cudaMemcpy (whose DMA from pageable memory may
  // still be in flight when it returns) or cudaMemset could land after the
  // first kernels on st read the state.
  if (e == cudaSuccess) e = cudaMemcpyAsync(z, hz.data(), nz2 * sizeof(double2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dd, hd0.data(), nd * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ii, hi0.data(), ni * sizeof(int), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && stamps)
    e = cudaMemsetAsync(stamps, 0, (size_t)(8 * scap + 1) * sizeof(unsigned long long), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host vectors may be released afterwards
  if (e != cudaSuccess) {
    if (st) cudaStreamDestroy(st);
    if (st2) cudaStreamDestroy(st2);
    cudaFree(blk); cudaFree(xpart); cudaFree(stamps);
    set_cuda_error("graph solve streams and state", e);
    return 1;
  }
  Engine<T>& eng = *io.eng;
  const cudaStream_t eng_st = eng.stream;
  MvArgs<T> mv;
  mv.x = vt; mv.x_rs = n; mv.y = atw; mv.y_rs = n; mv.io_full = 0;
  mv.adia = io.adia; mv.aoff = io.aoff; mv.a_rs = n; mv.a_full = 0; mv.conj = 0; mv.mask = S.live; mv.nrhs = R;
  // the MATVEC time of the iterations is estimated as mv_ms_per_rhs per RHS (the
  // kernels inside the graph are not timed)
  int rc = 0;
  eng.stream = st;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels_a = 0, kernels_b = 0;
  const double tol = io.tol;
  const int maxit = io.maxit;
  const unsigned gb = (unsigned)std::max<size_t>(1, std::min<size_t>(ceil_div(n, BT), std::max(1, 2368 / R)));
  if (!rc) {
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle h = 0;
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault);
    const unsigned long long c0 = launch_total();
    if (e == cudaSuccess) {
      // body of iteration k: its p/q/v step ran at the end of k-1 (or in the prologue)
      stamp(st, 0, 0);
      mv.x = vt; mv.y = atw; mv.mask = S.I;
      if (xpart) {  // vt^T A vt summed inside the last MATVEC pass
        mv.dot_out = ops.d_out; mv.dot_part = xpart; mv.dot_cnt = ops.d_cnt; mv.dot_k = 0;
      }
      rc = eng.matvec(mv);
      mv.dot_out = nullptr; mv.dot_part = nullptr; mv.dot_cnt = nullptr;
      if (!xpart) {
        BDot<T> sp{};
        sp.K = 1; sp.mode = 0; sp.a[0] = vt; sp.b[0] = atw; sp.conj[0] = 0;
        kb_dots<T><<<dim3(ops.nb, R), BT, 0, st>>>(n, sp, S.I, ops.d_part, ops.d_out, ops.d_cnt);
        note_launch();
      }
      stamp(st, 1, 0);
      k_qg_scalars<<<1, 256, 0, st>>>(R, S, ops.d_out);
      note_launch();
      stamp(st, 2, 0);
      kq_dsxr_pqv<C><<<dim3(ops.nb, R), BT, 0, st>>>(n, d, s, xs, r, p, q, vt, atw, S.co, S.I, ops.d_part,
                                                     ops.d_out, ops.d_cnt);
      note_launch();
      stamp(st, 3, 0);
      k_qg_post<<<1, 32, 0, st>>>(R, tol, S, ops.d_out, h);
      note_launch();
      stamp(st, 4, 0);
      kernels_a = launch_total() - c0;
      // IF node: the reliable-residual check
      e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &graph, &deps, &ndeps);
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t cnode = nullptr;
      if (e == cudaSuccess) e = cudaGraphAddNode(&cnode, graph, deps, ndeps, &cp);
      if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
      if (e == cudaSuccess) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        e = cudaStreamBeginCaptureToGraph(st2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          const unsigned long long c1 = launch_total();
          eng.stream = st2;
          MvArgs<T> ck = mv;
          ck.x = xs; ck.y = sy; ck.mask = S.CK;
          if (!rc) rc = eng.matvec(ck);
          BDot<T> dn{};
          dn.K = 2; dn.mode = 1; dn.a[0] = io.b; dn.b[0] = sy; dn.c[0] = r;
          kb_dots<T><<<dim3(ops.nb, R), BT, 0, st2>>>(n, dn, S.CK, ops.d_part, ops.d_out, ops.d_cnt);
          note_launch();
          k_qg_check<<<1, 256, 0, st2>>>(R, tol, S, ops.d_out);
          note_launch();
          kb_lin<C><<<dim3(gb, R), BT, 0, st2>>>(n, r, nullptr, io.b, S.one, sy, S.mone, S.RP);
          note_launch();
          kernels_b = launch_total() - c1;
          cudaGraph_t body_out = nullptr;
          e = cudaStreamEndCapture(st2, &body_out);
          eng.stream = st;
        }
      }
      if (e == cudaSuccess) {
        stamp(st, 5, 0);
        k_qg_next<<<1, 32, 0, st>>>(R, maxit, tol, S);
        note_launch();
        stamp(st, 6, 1);
        kernels_a += 1;
      }
    }
    cudaGraph_t g_out = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(st, &g_out);
    if (e == cudaSuccess) e = e2;
    graph = g_out;
    if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) { set_cuda_error("graph solve capture", e); rc = 1; }
  }
  // capture only recorded the launches: the counter counts executions below
  if (!rc) {
    // prologue: the first iteration's start and p/q/v step
    k_qg_begin<<<1, 256, 0, st>>>(R, maxit, tol, S);
    kq_pqv<C><<<dim3(ops.nb, R), BT, 0, st>>>(n, p, q, vt, atw, S.co, S.I, 2, ops.d_part, ops.d_out, ops.d_cnt);
    note_launch(2);
    int* h_active = nullptr;
    e = cudaMallocHost((void**)&h_active, sizeof(int));
    long long launches = 0;
    const long long cap = (long long)maxit + 64;  // every RHS stops at maxit; the loop is bounded
    while (e == cudaSuccess && launches < cap) {
      for (int k = 0; k < 4 && e == cudaSuccess; ++k, ++launches) e = cudaGraphLaunch(exec, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(h_active, S.active, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess || *h_active == 0) break;
    }
    int checks = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&checks, S.checks, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_cuda_error("graph solve", e); rc = 1; }
    note_launch((unsigned long long)launches * kernels_a + (unsigned long long)checks * kernels_b);
    if (stamps && e == cudaSuccess) {
      std::vector<unsigned long long> hs((size_t)8 * scap + 1);
      if (cudaMemcpy(hs.data(), stamps, hs.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost) ==
          cudaSuccess) {
        const long long nit = (long long)std::min<unsigned long long>(hs[(size_t)8 * scap], (unsigned long long)scap);
        double ph[7] = {0, 0, 0, 0, 0, 0, 0};
        long long cntv = 0;
        for (long long i = 0; i + 1 < nit; ++i) {
          const unsigned long long* a = &hs[(size_t)8 * i];
          for (int k = 0; k < 6; ++k) ph[k] += (double)(a[k + 1] - a[k]) * 1e-3;
          ph[6] += (double)(hs[(size_t)8 * (i + 1)] - a[6]) * 1e-3;
          ++cntv;
        }
        if (cntv > 0)
          std::printf("batched QMRCCG, %d RHS, %lld iterations (us per iteration): MATVEC + vt^T A vt %.1f | "
                      "scalars %.1f | d/s/x/r + p/q/v %.1f | residual bookkeeping %.1f | reliable-residual check "
                      "(IF node) %.1f | next-iteration start %.1f | gap %.1f\n",
                      R, cntv, ph[0] / cntv, ph[1] / cntv, ph[2] / cntv, ph[3] / cntv, ph[4] / cntv, ph[5] / cntv,
                      ph[6] / cntv);
      }
    }
    cudaFreeHost(h_active);
    if (!rc) {
      std::vector<double> hd(nd);
      std::vector<int> hi(ni);
      std::vector<double2> hz(nz2);
      e = cudaMemcpy(hd.data(), dd, nd * sizeof(double), cudaMemcpyDeviceToHost);
      if (e == cudaSuccess) e = cudaMemcpy(hi.data(), ii, ni * sizeof(int), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { set_cuda_error("graph solve state", e); rc = 1; }
      long long mv_rhs = 0;
      for (int i = 0; i < R && !rc; ++i) {
        resid[i] = hd[R + i];
        it[i] = hi[i]; live[i] = hi[R + i]; status[i] = hi[2 * R + i];
        mv_rhs += hi[3 * R + i] - nc[i];
        nc[i] = hi[3 * R + i];
      }
      io.matvec_rhs += mv_rhs;
      io.matvec_calls += (int)(launches + checks);
      io.matvec_ms += mv_ms_per_rhs * (double)mv_rhs;
    }
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  eng.stream = eng_st;
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cudaStreamDestroy(st2);
  cudaFree(blk);
  cudaFree(xpart);
  cudaFree(stamps);
  return rc;
}

// --------------------------------------------------------------------------
// QMRCCG (per RHS: solvers.cu solve_qmrccg, reference cu:434-443, cu:1071-1103)
template <typename T> int solve_batch_qmrccg(BatchIO<T>& io, BatchResult& res) {
  using C = cplx<T>;
  BCtx<T> c(io);
  BatchOps<T>& ops = c.ops;
  const int R = io.R;
  C *r = c.w(0), *p = c.w(1), *ap = c.w(2), *q = c.w(3), *d = c.w(4), *s = c.w(5);
  C *vt = c.w(6), *wt = c.w(7), *atw = c.w(8), *sy = c.w(9), *xs = io.x;
  const std::vector<double2> one = BCtx<T>::cst(R, 1.0), mone = BCtx<T>::cst(R, -1.0);
  res.itno.assign(R, 0); res.ncompte.assign(R, 0); res.status.assign(R, 0); res.tole.assign(R, 0.0);
  std::vector<int> live(R, 1);  // not failed, not converged
  std::vector<double> bnorm(R), resid(R);
  std::vector<Z> lambda(R), kappa(R), theta(R), gamma(R), ksi(R), rho(R), eps(R), mu(R), tau(R);
  // sym: the left Lanczos vectors equal the right ones (wt0 = vt0 = r0 and
  // A^T = A, so wt_k = vt_k and q_k = A p_k for every k): wt is not stored,
  // q is kept by its recurrence as A p, and one MATVEC (A vt) per iteration
  // remains.  Same iterates as the two-product form in exact arithmetic.
  const bool sym = io.sym != 0;
  std::vector<double2> o;
  const C* A1[3];
  const C* B1[3];
  int cj[3];
  // ||b|| and ||x0||: A x0 is formed only for a nonzero x0 (for x0 = 0 it is
  // exactly zero; the product still counts in NCOMPTE, as in the reference)
  A1[0] = io.b; B1[0] = io.b; cj[0] = 1;
  A1[1] = xs; B1[1] = xs; cj[1] = 1;
  if (ops.dots(2, A1, B1, cj, nullptr, o)) return 1;
  std::vector<int> x0nz(R, 0), x0z(R, 0);
  for (int i = 0; i < R; ++i) {
    bnorm[i] = std::sqrt(std::max(0.0, o[2 * i].x));
    if (bnorm[i] == 0.0) { res.status[i] = 52; live[i] = 0; }
    x0nz[i] = live[i] && o[2 * i + 1].x != 0.0;
    x0z[i] = live[i] && !x0nz[i];
  }
  const int* M = ops.mask(live);
  int rc = c.mv(xs, sy, x0nz);
  if (rc) return rc;
  if (any_of(x0z)) {
    ops.zero(sy, ops.mask(x0z));
    for (int i = 0; i < R; ++i) { c.nc[i] += x0z[i]; io.matvec_rhs += x0z[i]; }
  }
  ops.lin(r, nullptr, io.b, one.data(), sy, mone.data(), M);
  for (C* v : {p, ap, q, d, s, atw}) ops.zero(v, M);
  ops.copy(vt, r, M);
  if (!sym) ops.copy(wt, r, M);
  auto init_scalars = [&](const std::vector<int>& set) -> int {
    const int* Ms = ops.mask(set);
    if (sym) {
      const C* A2[2] = {vt, vt};
      const C* B2[2] = {vt, vt};
      const int c2[2] = {1, 0};
      std::vector<double2> o2, o1;
      if (ops.dots(2, A2, B2, c2, Ms, o2)) return 1;
      int rc2 = c.mv(vt, atw, set);
      if (rc2) return rc2;
      const C* A1b[1] = {vt};
      const C* B1b[1] = {atw};
      const int c1[1] = {0};
      if (ops.dots(1, A1b, B1b, c1, Ms, o1)) return 1;
      for (int i = 0; i < R; ++i) {
        if (!set[i]) continue;
        const double gn = std::sqrt(std::max(0.0, o2[2 * i].x));
        rho[i] = zd2(o2[2 * i + 1]);
        eps[i] = zd2(o1[i]);
        lambda[i] = 1.0; kappa[i] = -1.0; theta[i] = -1.0; gamma[i] = gn; ksi[i] = gn; mu[i] = 0.0;
        if (rho[i] == Z(0.0) || gamma[i] == Z(0.0)) { res.status[i] = 55; live[i] = 0; continue; }
        tau[i] = eps[i] / rho[i];
      }
      return 0;
    }
    const C* A3[3] = {vt, wt, vt};
    const C* B3[3] = {vt, wt, wt};
    const int c3[3] = {1, 1, 0};
    std::vector<double2> o3, o1;
    if (ops.dots(3, A3, B3, c3, Ms, o3)) return 1;
    int rc2 = c.mv(wt, atw, set);
    if (rc2) return rc2;
    const C* A1b[1] = {vt};
    const C* B1b[1] = {atw};
    const int c1[1] = {0};
    if (ops.dots(1, A1b, B1b, c1, Ms, o1)) return 1;
    for (int i = 0; i < R; ++i) {
      if (!set[i]) continue;
      const double gn = std::sqrt(std::max(0.0, o3[3 * i].x)), kn = std::sqrt(std::max(0.0, o3[3 * i + 1].x));
      rho[i] = zd2(o3[3 * i + 2]);
      eps[i] = zd2(o1[i]);
      lambda[i] = 1.0; kappa[i] = -1.0; theta[i] = -1.0; gamma[i] = gn; ksi[i] = kn; mu[i] = 0.0;
      if (rho[i] == Z(0.0) || gamma[i] == Z(0.0) || ksi[i] == Z(0.0)) { res.status[i] = 55; live[i] = 0; continue; }
      tau[i] = eps[i] / rho[i];
    }
    return 0;
  };
  if ((rc = init_scalars(live))) return rc;
  {
    const C* Ar[1] = {r};
    const int c1[1] = {1};
    if (ops.dots(1, Ar, Ar, c1, ops.mask(live), o)) return 1;
    for (int i = 0; i < R; ++i)
      if (live[i]) resid[i] = std::sqrt(std::max(0.0, o[i].x)) / bnorm[i];
  }
  std::vector<int> it(R, 0);
  const bool use_graph = io.graph && sym && io.replace;
  if (use_graph) {
    C* wv[10] = {c.w(0), c.w(1), c.w(2), c.w(3), c.w(4), c.w(5), c.w(6), c.w(7), c.w(8), c.w(9)};
    std::vector<Z> sc[9] = {gamma, ksi, rho, eps, mu, tau, lambda, kappa, theta};
    // MATVEC time per RHS from the latest timed MATVEC of the setup (A vt0)
    float t = 0.f;
    cudaStreamSynchronize(ops.stream);
    if (!c.ev.empty()) cudaEventElapsedTime(&t, c.ev.back().first, c.ev.back().second);
    const double per_rhs = c.last_cnt > 0 ? (double)t / c.last_cnt : 0.0;
    if ((rc = qmr_graph_loop<T>(io, ops, c.nc, wv, xs, sc, bnorm, resid, it, live, res.status, per_rhs))) return rc;
  }
  for (; !use_graph;) {
    std::vector<int> I(R, 0);
    for (int i = 0; i < R; ++i) I[i] = live[i] && it[i] < io.maxit && resid[i] > io.tol;
    if (!any_of(I)) break;
    for (int i = 0; i < R; ++i) it[i] += I[i];
    const int* MI = ops.mask(I);
    std::vector<double2> cmu(R), cgam(R), cq(R), cksi(R), ctg(R), ctk(R), cth(R), cka(R);
    for (int i = 0; i < R; ++i) {
      if (!I[i]) continue;
      cmu[i] = dz(-mu[i]); cgam[i] = dz(1.0 / gamma[i]);
      cq[i] = dz(-(gamma[i] * mu[i]) / ksi[i]); cksi[i] = dz(1.0 / ksi[i]);
    }
    for (int i = 0; i < R; ++i) {
      if (!I[i]) continue;
      ctg[i] = dz(-(tau[i] / gamma[i]));
      ctk[i] = dz(-(tau[i] / ksi[i]));
    }
    const C* Ap = sym ? q : ap;  // A p
    const C* W = sym ? vt : wt;  // left Lanczos vector
    std::vector<double2> o3, o1;
    if (sym) {
      // one fused pass: p, q (= A p), vt and the sums |vt|^2, vt^T vt
      if (ops.qmr_pqv(p, q, vt, atw, cmu.data(), cgam.data(), cq.data(), cksi.data(), ctg.data(), MI)) return 1;
    } else {
      ops.lin(p, cmu.data(), vt, cgam.data(), nullptr, nullptr, MI);
      ops.lin(q, cq.data(), atw, cksi.data(), nullptr, nullptr, MI);
      if ((rc = c.mv(p, ap, I))) return rc;
      ops.lin(vt, ctg.data(), Ap, one.data(), nullptr, nullptr, MI);
      ops.lin(wt, ctk.data(), q, one.data(), nullptr, nullptr, MI);
      const C* A3[3] = {vt, W, vt};
      const C* B3[3] = {vt, W, W};
      const int c3[3] = {1, 1, 0};
      if (ops.dots(3, A3, B3, c3, MI, o3)) return 1;
    }
    if ((rc = c.mv(W, atw, I))) return rc;
    {
      const C* A1b[1] = {vt};
      const C* B1b[1] = {atw};
      const int c1[1] = {0};
      if (ops.dots(1, A1b, B1b, c1, MI, o1)) return 1;
    }
    if (sym) {
      o3.assign((size_t)3 * R, make_double2(0, 0));
      for (int i = 0; i < R; ++i) {
        if (!I[i]) continue;
        o3[3 * i] = o3[3 * i + 1] = ops.slot(i, 2);
        o3[3 * i + 2] = ops.slot(i, 3);
      }
    }
    for (int i = 0; i < R; ++i) {
      if (!I[i]) continue;
      const Z gamma0 = gamma[i], ksi0 = ksi[i], rho0 = rho[i], tau0 = tau[i], kappa0 = kappa[i];
      gamma[i] = std::sqrt(std::max(0.0, o3[3 * i].x));
      ksi[i] = std::sqrt(std::max(0.0, o3[3 * i + 1].x));
      rho[i] = zd2(o3[3 * i + 2]);
      eps[i] = zd2(o1[i]);
      int st = 0;
      if (gamma[i] == Z(0.0)) st = 6;
      else if (ksi[i] == Z(0.0)) st = 7;
      const Z den = gamma[i] * tau[i] * rho0;
      if (!st && den == Z(0.0)) st = 12;
      if (!st) { mu[i] = gamma0 * ksi0 * rho[i] / den; if (rho[i] == Z(0.0)) st = 13; }
      if (!st) {
        tau[i] = eps[i] / rho[i] - gamma[i] * mu[i];
        const double at0 = std::norm(tau0), ag = std::norm(gamma[i]);
        const Z den2 = lambda[i] * at0 + ag;
        if (den2 == Z(0.0)) st = 14;
        else {
          theta[i] = ((1.0 - lambda[i]) * at0) / den2;
          kappa[i] = -(gamma0 * std::conj(tau0) * kappa0) / den2;
          lambda[i] = (lambda[i] * at0) / den2;
        }
      }
      if (st) { res.status[i] = 58; live[i] = 0; I[i] = 0; }
      cth[i] = dz(theta[i]);
      cka[i] = dz(kappa[i]);
    }
    MI = ops.mask(I);
    if (sym) {
      // one fused pass: d, s, x, r and |r|^2
      if (ops.qmr_dsxr(d, s, xs, r, p, Ap, cth.data(), cka.data(), MI, o)) return 1;
    } else {
      ops.lin(d, cth.data(), p, cka.data(), nullptr, nullptr, MI);
      ops.lin(s, cth.data(), Ap, cka.data(), nullptr, nullptr, MI);
      ops.lin(xs, one.data(), d, one.data(), nullptr, nullptr, MI);
      ops.lin(r, one.data(), s, mone.data(), nullptr, nullptr, MI);
      const C* Ar[1] = {r};
      const int c1[1] = {1};
      if (ops.dots(1, Ar, Ar, c1, MI, o)) return 1;
    }
    for (int i = 0; i < R; ++i)
      if (I[i]) resid[i] = std::sqrt(std::max(0.0, o[i].x)) / bnorm[i];
    std::vector<int> CK(R, 0);
    for (int i = 0; i < R; ++i) CK[i] = I[i] && ((it[i] % 20) == 0 || resid[i] <= io.tol);
    if (any_of(CK)) {
      if ((rc = c.mv(xs, sy, CK))) return rc;
      std::vector<double2> nn;
      if (ops.diff_norms(io.b, sy, r, ops.mask(CK), nn)) return 1;
      std::vector<int> RS(R, 0), RP(R, 0);
      for (int i = 0; i < R; ++i) {
        if (!CK[i]) continue;
        const double tr = std::sqrt(std::max(0.0, nn[2 * i].x)), gapn = std::sqrt(std::max(0.0, nn[2 * i + 1].x));
        const double tres = tr / bnorm[i];
        const double gap = tr > 0.0 ? gapn / tr : (gapn == 0.0 ? 0.0 : INFINITY);
        const bool conv = tres <= io.tol;
        const bool rest = gap >= 1.0e-3 || (resid[i] <= io.tol && !conv);
        if (conv) { resid[i] = tres; live[i] = 0; continue; }
        if (rest && io.replace) { RP[i] = 1; resid[i] = tres; }
        else if (rest) { RS[i] = 1; resid[i] = tres; }
      }
      if (any_of(RP)) {
        // residual replacement: r = b - A x; the Lanczos vectors and scalars
        // do not depend on r, so the iterates are unchanged
        ops.lin(r, nullptr, io.b, one.data(), sy, mone.data(), ops.mask(RP));
      }
      if (any_of(RS)) {
        const int* MR = ops.mask(RS);
        ops.lin(sy, mone.data(), io.b, one.data(), nullptr, nullptr, MR);  // sy = b - A x
        ops.copy(r, sy, MR);
        for (C* v : {p, ap, q, d, s, atw}) ops.zero(v, MR);
        ops.copy(vt, sy, MR);
        if (!sym) ops.copy(wt, sy, MR);
        if ((rc = init_scalars(RS))) return rc;
      }
    }
  }
  // RHS that stopped at MAXIT: one final true residual (cu:1099)
  std::vector<int> F(R, 0);
  for (int i = 0; i < R; ++i) F[i] = res.status[i] == 0 && resid[i] > io.tol;
  if (any_of(F)) {
    if ((rc = c.mv(xs, sy, F))) return rc;
    std::vector<double2> nn;
    if (ops.diff_norms(io.b, sy, r, ops.mask(F), nn)) return 1;
    for (int i = 0; i < R; ++i)
      if (F[i]) resid[i] = std::sqrt(std::max(0.0, nn[2 * i].x)) / bnorm[i];
  }
  c.finish_timing();
  for (int i = 0; i < R; ++i) { res.itno[i] = it[i]; res.tole[i] = resid[i]; res.ncompte[i] = c.nc[i]; }
  return 0;
}

// --------------------------------------------------------------------------
// Device-driven PBCGS2 iteration (residual replacement), captured in a CUDA
// graph: the host-driven recurrence of solve_batch_pbcgs2 below, with its
// per-RHS FP64 scalars (rho, alpha, beta, omega, the 3 x 3 minimal-residual
// system of the BiCGStab(2) step, the reliable-update tests) in single-thread
// kernels on state held on the GPU.  Two IF conditional nodes hold the
// reliable-residual check (every 20 iterations and at convergence) and the
// reliable update of the solution (cu:474), armed on the device only when some
// RHS needs them.  The host launches the graph repeatedly and reads the active
// count every few launches.
struct PGState {
  double2 *alpha, *omega, *sigma, *rho0, *rho1, *beta;
  double2* co;           // [7][R]: -beta, alpha, -alpha, y1, y2, -y1, -y2
  double2 *one, *mone;   // [R]
  double *rnrm0, *rnrm, *mxx, *mxr, *resid;
  int *it, *live, *status, *nc, *I, *CK, *RP, *RC, *XD, *RCMP, *XPDT;
  int *active, *checks, *updates, *loops;  // [1] each
};

__device__ __forceinline__ double2 dconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double dabs(double2 a) { return hypot(a.x, a.y); }

// start of an iteration: I = live, resid > tol, it < maxit; rho0 = -(omega rho0)
__global__ void k_pg_begin(int R, int maxit, double tol, PGState S) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    const int on = S.live[r] && S.resid[r] > tol && S.it[r] < maxit;
    S.I[r] = on;
    if (!on) continue;
    S.it[r] += 1;
    S.rho0[r] = dsc(-1.0, dmul(S.omega[r], S.rho0[r]));
  }
}

// rho1 = rr^H r_{k-1} (out slot 0), beta and the coefficient -beta of the u update
__global__ void k_pg_rho(int R, PGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.I[r]) continue;
    const double2 rho1 = out[(size_t)r * 8];
    S.rho1[r] = rho1;
    if (dz0(S.rho0[r])) { S.status[r] = 95; S.live[r] = 0; S.I[r] = 0; continue; }
    const double2 beta = dmul(S.alpha[r], ddiv(rho1, S.rho0[r]));
    S.beta[r] = beta;
    S.rho0[r] = rho1;
    S.co[r] = dsc(-1.0, beta);
    S.nc[r] += 1;  // the MATVEC u_{k-1} -> u_k that follows
  }
}

// sigma = rr^H u_k (out slot 0), alpha and the coefficients alpha, -alpha
__global__ void k_pg_sigma(int R, PGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.I[r]) continue;
    const double2 sg = out[(size_t)r * 8];
    S.sigma[r] = sg;
    if (dz0(sg)) { S.status[r] = 98; S.live[r] = 0; S.I[r] = 0; continue; }
    const double2 al = ddiv(S.rho1[r], sg);
    S.alpha[r] = al;
    S.co[R + r] = al;
    S.co[2 * R + r] = dsc(-1.0, al);
    S.nc[r] += 1;  // the MATVEC r_{k-1} -> r_k that follows
  }
}

// |r_0| (out slot 0) and its running maxima
__global__ void k_pg_rnrm(int R, PGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.I[r]) continue;
    const double v = sqrt(fmax(0.0, out[(size_t)r * 8].x));
    S.rnrm[r] = v;
    S.mxx[r] = fmax(S.mxx[r], v);
    S.mxr[r] = fmax(S.mxr[r], v);
  }
}

// the BiCGStab(2) minimal-residual step from the Gram matrix of r_0, r_1, r_2
// (out slots 0..5: (0,0), (1,0), (1,1), (2,0), (2,1), (2,2), conjugated first
// argument), as in the host form (cu:1168-1278 via solvers.cu)
__global__ void k_pg_gram(int R, PGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.I[r]) continue;
    const double2* o = out + (size_t)r * 8;
    double2 Zm[3][3];
    Zm[0][0] = o[0]; Zm[1][0] = o[1]; Zm[1][1] = o[2];
    Zm[2][0] = o[3]; Zm[2][1] = o[4]; Zm[2][2] = o[5];
    Zm[0][1] = dconj(Zm[1][0]); Zm[0][2] = dconj(Zm[2][0]); Zm[1][2] = dconj(Zm[2][1]);
    auto matv = [&](const double2* v, double2* w) {
      for (int a = 0; a < 3; ++a) {
        w[a] = make_double2(0.0, 0.0);
        for (int b = 0; b < 3; ++b) w[a] = dadd(w[a], dmul(Zm[a][b], v[b]));
      }
    };
    auto inner = [](const double2* a, const double2* b) {
      double2 s = make_double2(0.0, 0.0);
      for (int k = 0; k < 3; ++k) s = dadd(s, dmul(dconj(a[k]), b[k]));
      return s;
    };
    bool fail = dz0(Zm[1][1]);
    double2 y0[3], yl[3], zy0[3], zyl[3];
    double k0 = 0.0, kl = 0.0;
    if (!fail) {
      y0[0] = make_double2(-1.0, 0.0); y0[1] = ddiv(Zm[1][0], Zm[1][1]); y0[2] = make_double2(0.0, 0.0);
      yl[0] = make_double2(0.0, 0.0); yl[1] = ddiv(Zm[1][2], Zm[1][1]); yl[2] = make_double2(-1.0, 0.0);
      matv(y0, zy0);
      matv(yl, zyl);
      k0 = sqrt(dabs(inner(y0, zy0)));
      kl = sqrt(dabs(inner(yl, zyl)));
      fail = k0 == 0.0 || kl == 0.0;
    }
    double2 vr = make_double2(0.0, 0.0);
    double avr = 0.0;
    if (!fail) {
      const double2 q = inner(yl, zy0);
      const double den = k0 * kl;
      vr = make_double2(q.x / den, q.y / den);
      avr = dabs(vr);
      fail = avr == 0.0;
    }
    if (fail) { S.status[r] = 102; S.live[r] = 0; S.I[r] = 0; continue; }
    const double s1 = fmax(avr, 0.7) / avr, s2 = k0 / kl;
    const double2 fac = dsc(s2, dsc(s1, vr));
    for (int a = 0; a < 3; ++a) {
      const double2 f = dmul(fac, yl[a]);
      y0[a] = make_double2(y0[a].x - f.x, y0[a].y - f.y);
    }
    S.omega[r] = y0[2];
    matv(y0, zy0);
    const double rn = sqrt(dabs(inner(y0, zy0)));
    S.rnrm[r] = rn;
    S.mxx[r] = fmax(S.mxx[r], rn);
    S.mxr[r] = fmax(S.mxr[r], rn);
    S.co[3 * R + r] = y0[1];
    S.co[4 * R + r] = y0[2];
    S.co[5 * R + r] = dsc(-1.0, y0[1]);
    S.co[6 * R + r] = dsc(-1.0, y0[2]);
    const double r0n = S.rnrm0[r];
    const int xpdt = rn < 1.0e-2 * r0n && r0n < S.mxx[r];
    S.XPDT[r] = xpdt;
    S.RCMP[r] = (rn < 1.0e-2 * S.mxr[r] && r0n < S.mxr[r]) || xpdt;
    S.resid[r] = r0n > 0.0 ? rn / r0n : 0.0;
  }
}

// reliable-residual check mask (every 20 iterations and at convergence) and its IF condition
__global__ void k_pg_post(int R, double tol, PGState S, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  int any = 0;
  for (int r = 0; r < R; ++r) {
    const int ck = S.I[r] && ((S.it[r] % 20) == 0 || S.resid[r] <= tol);
    S.CK[r] = ck;
    S.RP[r] = 0;
    if (ck) S.nc[r] += 1;
    any |= ck;
  }
  if (any) *S.checks += 1;
  cudaGraphSetConditional(h, any ? 1u : 0u);
}

// decisions of the check from |b' - A x|^2, |b' - A x - r_0|^2 (b' the shifted RHS)
__global__ void k_pg_check(int R, double tol, PGState S, const double2* out) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.CK[r]) continue;
    const double tr = sqrt(fmax(0.0, out[(size_t)r * 8].x)), gapn = sqrt(fmax(0.0, out[(size_t)r * 8 + 1].x));
    const double tres = tr / S.rnrm0[r];
    const double gap = tr > 0.0 ? gapn / tr : (gapn == 0.0 ? 0.0 : INFINITY);
    const bool conv = tres <= tol;
    const bool rest = gap >= 1.0e-3 || (S.resid[r] <= tol && !conv);
    if (conv) { S.resid[r] = tres; S.live[r] = 0; S.I[r] = 0; continue; }
    if (rest) {
      S.RP[r] = 1;
      S.resid[r] = tres;
      S.rnrm[r] = tres * S.rnrm0[r];
      S.mxr[r] = fmax(S.mxr[r], S.rnrm[r]);
    }
  }
}

// reliable-update masks (RC: recompute r_0; XD: also shift the solution) and their IF condition
__global__ void k_pg_rc(int R, PGState S, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  int any = 0;
  for (int r = 0; r < R; ++r) {
    const int rc = S.I[r] && S.RCMP[r];
    S.RC[r] = rc;
    S.XD[r] = rc && S.XPDT[r];
    if (rc) S.nc[r] += 1;
    any |= rc;
  }
  if (any) *S.updates += 1;
  cudaGraphSetConditional(h, any ? 1u : 0u);
}

__global__ void k_pg_rcpost(int R, PGState S) {
  for (int r = threadIdx.x; r < R; r += blockDim.x) {
    if (!S.RC[r]) continue;
    S.mxr[r] = S.rnrm[r];
    if (S.XD[r]) S.mxx[r] = S.rnrm[r];
  }
}

// RHS that will run another iteration
__global__ void k_pg_count(int R, int maxit, double tol, PGState S) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int r = 0; r < R; ++r) c += S.live[r] && S.resid[r] > tol && S.it[r] < maxit;
  *S.active = c;
  *S.loops += 1;
}
// the same as the last kernel of an iteration that runs as the body of a WHILE
// node: the loop continues while some RHS is active (each pass raises `it` of
// every active RHS, so it ends after at most maxit passes)
__global__ void k_pg_count_while(int R, int maxit, double tol, PGState S, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int r = 0; r < R; ++r) c += S.live[r] && S.resid[r] > tol && S.it[r] < maxit;
  *S.active = c;
  *S.loops += 1;
  cudaGraphSetConditional(h, c > 0 ? 1u : 0u);
}

// host copy of the PBCGS2 state handed between the host-driven and the graph-driven iterations
struct PGHost {
  std::vector<Z> alpha, omega, sigma, rho0, rho1, beta;
  std::vector<double> rnrm0, rnrm, mxx, mxr, resid;
  std::vector<int> it, live, status;
};

// One target's device-driven PBCGS2 iterations (residual replacement) as a
// graph body: init() moves the host state hs onto the GPU, capture() records one
// iteration into the capture its stream st has joined (its IF-node bodies on
// st2), pg_run() launches the captured iteration until no RHS is active, and
// readback() brings the state back; w: rr, r0, r1, r2, u0, u1, u2, XP, BP, X, sy.
template <typename T> struct PGGraph {
  using C = cplx<T>;
  BatchIO<T>* io = nullptr;
  BatchOps<T>* ops = nullptr;
  std::vector<int>* nc = nullptr;
  PGHost* hs = nullptr;
  C* w[11] = {};
  double mv_ms_per_rhs = 0.0;
  int R = 0, n = 0;
  size_t nz2 = 0, nd = 0, ni = 0;
  unsigned char* blk = nullptr;
  double* dd = nullptr;
  int* ii = nullptr;
  PGState S{};
  cudaStream_t st = nullptr, st2 = nullptr, stw = nullptr, eng_st = nullptr;
  unsigned long long kernels_a = 0, kernels_b = 0, kernels_c = 0;
  long long launches = 0;  // set by pg_run

  int init(BatchIO<T>& io_, BatchOps<T>& ops_, std::vector<int>& nc_, C* const* w_, PGHost& hs_, double per_rhs) {
    io = &io_; ops = &ops_; nc = &nc_; hs = &hs_; mv_ms_per_rhs = per_rhs;
    for (int k = 0; k < 11; ++k) w[k] = w_[k];
    R = io->R; n = io->n;
    nz2 = (size_t)(6 + 7 + 2) * R; nd = (size_t)5 * R; ni = (size_t)11 * R + 4;
    cudaError_t e = cudaMalloc((void**)&blk, nz2 * sizeof(double2) + nd * sizeof(double) + ni * sizeof(int));
    if (e != cudaSuccess) { set_cuda_error("graph solve state", e); return 1; }
    double2* z = reinterpret_cast<double2*>(blk);
    double2** zp[6] = {&S.alpha, &S.omega, &S.sigma, &S.rho0, &S.rho1, &S.beta};
    for (int k = 0; k < 6; ++k) *zp[k] = z + (size_t)k * R;
    S.co = z + (size_t)6 * R;
    S.one = z + (size_t)13 * R;
    S.mone = z + (size_t)14 * R;
    dd = reinterpret_cast<double*>(z + nz2);
    double** dp[5] = {&S.rnrm0, &S.rnrm, &S.mxx, &S.mxr, &S.resid};
    for (int k = 0; k < 5; ++k) *dp[k] = dd + (size_t)k * R;
    ii = reinterpret_cast<int*>(dd + nd);
    int** ip[11] = {&S.it, &S.live, &S.status, &S.nc, &S.I, &S.CK, &S.RP, &S.RC, &S.XD, &S.RCMP, &S.XPDT};
    for (int k = 0; k < 11; ++k) *ip[k] = ii + (size_t)k * R;
    S.active = ii + (size_t)11 * R;
    S.checks = S.active + 1;
    S.updates = S.active + 2;
    S.loops = S.active + 3;
    std::vector<double2> hz(nz2, make_double2(0, 0));
    const std::vector<Z>* zs[6] = {&hs->alpha, &hs->omega, &hs->sigma, &hs->rho0, &hs->rho1, &hs->beta};
    for (int k = 0; k < 6; ++k)
      for (int i = 0; i < R; ++i) hz[(size_t)k * R + i] = dz((*zs[k])[i]);
    for (int i = 0; i < R; ++i) { hz[(size_t)13 * R + i] = make_double2(1, 0); hz[(size_t)14 * R + i] = make_double2(-1, 0); }
    std::vector<double> hd0(nd);
    const std::vector<double>* ds[5] = {&hs->rnrm0, &hs->rnrm, &hs->mxx, &hs->mxr, &hs->resid};
    for (int k = 0; k < 5; ++k)
      for (int i = 0; i < R; ++i) hd0[(size_t)k * R + i] = (*ds[k])[i];
    std::vector<int> hi0(ni, 0);
    for (int i = 0; i < R; ++i) {
      hi0[i] = hs->it[i]; hi0[R + i] = hs->live[i]; hi0[2 * R + i] = hs->status[i]; hi0[3 * R + i] = (*nc)[i];
    }
    cudaStreamSynchronize(ops->stream);
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stw, cudaStreamNonBlocking);
    // uploads ordered on st (see qmr_graph_loop)
    if (e == cudaSuccess) e = cudaMemcpyAsync(z, hz.data(), nz2 * sizeof(double2), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dd, hd0.data(), nd * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ii, hi0.data(), ni * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { set_cuda_error("graph solve streams and state", e); return 1; }
    eng_st = io->eng->stream;
    return 0;
  }

  // one iteration into the capture stream st has joined; hwhile: the WHILE
  // node whose body this is (0: none, the host relaunches the graph)
  int capture(cudaGraphConditionalHandle hwhile = 0) {
    const int R_ = R, n_ = n;
    Engine<T>& eng = *io->eng;
    C *rr = w[0], *r[3] = {w[1], w[2], w[3]}, *u[3] = {w[4], w[5], w[6]}, *XP = w[7], *BP = w[8], *X = w[9],
      *sy = w[10];
    MvArgs<T> mv;
    mv.x_rs = n_; mv.y_rs = n_; mv.io_full = 0;
    mv.adia = io->adia; mv.aoff = io->aoff; mv.a_rs = n_; mv.a_full = 0; mv.conj = 0; mv.nrhs = R_;
    const double tol = io->tol;
    const int maxit = io->maxit;
    const unsigned gb = (unsigned)std::max<size_t>(1, std::min<size_t>(ceil_div(n_, BT), std::max(1, 2368 / R_)));
    BatchOps<T>& op = *ops;
    auto lin = [&](cudaStream_t s_, C* d, const double2* cd, const C* a, const double2* ca, const C* b,
                   const double2* cb, const int* m) {
      kb_lin<C><<<dim3(gb, R_), BT, 0, s_>>>(n_, d, cd, a, ca, b, cb, m);
      note_launch();
    };
    auto dots = [&](cudaStream_t s_, int K, const C* const* a, const C* const* b, const int* m) {
      BDot<T> sp{};
      sp.K = K; sp.mode = 0;
      for (int k = 0; k < K; ++k) { sp.a[k] = a[k]; sp.b[k] = b[k]; sp.conj[k] = 1; }
      kb_dots<T><<<dim3(op.nb, R_), BT, 0, s_>>>(n_, sp, m, op.d_part, op.d_out, op.d_cnt);
      note_launch();
    };
    auto matvec = [&](const C* in, C* out, const int* m) {
      mv.x = in; mv.y = out; mv.mask = m;
      return eng.matvec(mv);
    };
    // an IF node at the capture point of st whose body is captured on st2 by body()
    auto if_node = [&](cudaGraphConditionalHandle h, auto body) -> cudaError_t {
      cudaStreamCaptureStatus cs;
      cudaGraph_t g = nullptr;
      const cudaGraphNode_t* deps = nullptr;
      size_t ndeps = 0;
      cudaError_t e_ = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      cudaGraphNode_t cnode = nullptr;
      if (e_ == cudaSuccess) e_ = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp);
      if (e_ == cudaSuccess) e_ = cudaStreamUpdateCaptureDependencies(st, &cnode, 1, cudaStreamSetCaptureDependencies);
      if (e_ != cudaSuccess) return e_;
      e_ = cudaStreamBeginCaptureToGraph(st2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal);
      if (e_ != cudaSuccess) return e_;
      eng.stream = st2;
      body();
      eng.stream = st;
      cudaGraph_t body_out = nullptr;
      return cudaStreamEndCapture(st2, &body_out);
    };
    int rc = 0;
    eng.stream = st;
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle hck = 0, hrc = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps);
    if (e == cudaSuccess && cs != cudaStreamCaptureStatusActive) e = cudaErrorStreamCaptureInvalidated;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hck, g, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hrc, g, 0, cudaGraphCondAssignDefault);
    unsigned long long c0 = launch_total();
    if (e == cudaSuccess) {
      k_pg_begin<<<1, 256, 0, st>>>(R_, maxit, tol, S);
      note_launch();
      for (int k = 1; k <= 2 && !rc; ++k) {
        {
          const C* A1[1] = {rr};
          const C* B1[1] = {r[k - 1]};
          dots(st, 1, A1, B1, S.I);
        }
        k_pg_rho<<<1, 256, 0, st>>>(R_, S, op.d_out);
        note_launch();
        for (int j = 0; j < k; ++j) lin(st, u[j], S.co, r[j], S.one, nullptr, nullptr, S.I);
        if ((rc = matvec(u[k - 1], u[k], S.I))) break;
        {
          const C* A1[1] = {rr};
          const C* B1[1] = {u[k]};
          dots(st, 1, A1, B1, S.I);
        }
        k_pg_sigma<<<1, 256, 0, st>>>(R_, S, op.d_out);
        note_launch();
        lin(st, X, S.one, u[0], S.co + R_, nullptr, nullptr, S.I);
        for (int j = 0; j < k; ++j) lin(st, r[j], S.one, u[j + 1], S.co + 2 * R_, nullptr, nullptr, S.I);
        if ((rc = matvec(r[k - 1], r[k], S.I))) break;
        {
          const C* A1[1] = {r[0]};
          dots(st, 1, A1, A1, S.I);
        }
        k_pg_rnrm<<<1, 256, 0, st>>>(R_, S, op.d_out);
        note_launch();
      }
      if (!rc) {
        const C* A6[6] = {r[0], r[1], r[1], r[2], r[2], r[2]};
        const C* B6[6] = {r[0], r[0], r[1], r[0], r[1], r[2]};
        dots(st, 6, A6, B6, S.I);
        k_pg_gram<<<1, 64, 0, st>>>(R_, S, op.d_out);
        note_launch();
        lin(st, u[0], S.one, u[1], S.co + 5 * R_, u[2], S.co + 6 * R_, S.I);
        lin(st, X, S.one, r[0], S.co + 3 * R_, r[1], S.co + 4 * R_, S.I);
        lin(st, r[0], S.one, r[1], S.co + 5 * R_, r[2], S.co + 6 * R_, S.I);
        k_pg_post<<<1, 32, 0, st>>>(R_, tol, S, hck);
        note_launch();
        kernels_a = launch_total() - c0;
        // IF node 1: the reliable-residual check with residual replacement
        const unsigned long long c1 = launch_total();
        e = if_node(hck, [&]() {
          if (!rc) rc = matvec(X, sy, S.CK);
          BDot<T> dn{};
          dn.K = 2; dn.mode = 1; dn.a[0] = BP; dn.b[0] = sy; dn.c[0] = r[0];
          kb_dots<T><<<dim3(op.nb, R_), BT, 0, st2>>>(n_, dn, S.CK, op.d_part, op.d_out, op.d_cnt);
          note_launch();
          k_pg_check<<<1, 256, 0, st2>>>(R_, tol, S, op.d_out);
          note_launch();
          lin(st2, r[0], nullptr, BP, S.one, sy, S.mone, S.RP);
        });
        kernels_b = launch_total() - c1;
        if (e == cudaSuccess) {
          const unsigned long long c2 = launch_total();
          k_pg_rc<<<1, 32, 0, st>>>(R_, S, hrc);
          note_launch();
          kernels_a += launch_total() - c2;
          // IF node 2: the reliable update of r_0 (and of the solution shift)
          const unsigned long long c3 = launch_total();
          e = if_node(hrc, [&]() {
            if (!rc) rc = matvec(X, sy, S.RC);
            lin(st2, r[0], nullptr, BP, S.one, sy, S.mone, S.RC);
            lin(st2, XP, S.one, X, S.one, nullptr, nullptr, S.XD);
            lin(st2, X, nullptr, nullptr, nullptr, nullptr, nullptr, S.XD);
            lin(st2, BP, nullptr, r[0], S.one, nullptr, nullptr, S.XD);
            k_pg_rcpost<<<1, 256, 0, st2>>>(R_, S);
            note_launch();
          });
          kernels_c = launch_total() - c3;
        }
        if (e == cudaSuccess) {
          if (hwhile) k_pg_count_while<<<1, 32, 0, st>>>(R_, maxit, tol, S, hwhile);
          else k_pg_count<<<1, 32, 0, st>>>(R_, maxit, tol, S);
          note_launch();
          kernels_a += 1;
        }
      }
    }
    eng.stream = eng_st;
    if (e != cudaSuccess) { set_cuda_error("graph solve capture", e); return 1; }
    return rc;
  }

  // state back to the host after pg_run
  int readback() {
    std::vector<double> hd(nd);
    std::vector<int> hi(ni);
    cudaError_t e = cudaMemcpy(hd.data(), dd, nd * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hi.data(), ii, ni * sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { set_cuda_error("graph solve state", e); return 1; }
    const int checks = hi[(size_t)11 * R + 1], updates = hi[(size_t)11 * R + 2];
    launches = hi[(size_t)11 * R + 3];  // iterations run by the graph
    note_launch((unsigned long long)launches * kernels_a + (unsigned long long)checks * kernels_b +
                (unsigned long long)updates * kernels_c);
    long long mv_rhs = 0;
    for (int i = 0; i < R; ++i) {
      hs->resid[i] = hd[(size_t)4 * R + i];
      hs->it[i] = hi[i]; hs->live[i] = hi[R + i]; hs->status[i] = hi[2 * R + i];
      mv_rhs += hi[3 * R + i] - (*nc)[i];
      (*nc)[i] = hi[3 * R + i];
    }
    io->matvec_rhs += mv_rhs;
    io->matvec_calls += (int)(4 * launches + checks + updates);
    io->matvec_ms += mv_ms_per_rhs * (double)mv_rhs;
    return 0;
  }

  void release() {
    if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); }
    if (st2) cudaStreamDestroy(st2);
    if (stw) cudaStreamDestroy(stw);
    cudaFree(blk);
    st = st2 = stw = nullptr;
    blk = nullptr;
  }
};

// sum of the active-RHS counts of every branch
__global__ void k_pg_sum_active(int* const* act, int nb, int* out) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int b = 0; b < nb; ++b) c += *act[b];
  *out = c;
}

// One CUDA graph whose branches are the iterations of the given targets
// (independent of one another: fork from a root stream, join back).  With one
// target the graph is one iteration, launched once per Krylov step until no
// RHS is active (the host reads the active count every 4 launches).  With
// several, each branch is a WHILE node whose body is that target's iteration
// and whose condition its last kernel sets (some RHS still active): every
// target iterates on the device at its own pace, and the host launches the
// graph once.  Every pass raises the iteration count of each active RHS, so a
// branch ends after at most its maxit passes; the host relaunches (bounded)
// only if some branch is still active afterwards.
template <typename T> int pg_run(const std::vector<PGGraph<T>*>& gs) {
  if (gs.empty()) return 0;
  const int nb = (int)gs.size();
  const bool loops = nb > 1;
  cudaStream_t root = nullptr;
  int** d_act = nullptr;
  int* d_sum = nullptr;
  int* h_sum = nullptr;
  std::vector<cudaEvent_t> evs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int rc = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_act, (size_t)nb * sizeof(int*) + sizeof(int));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h_sum, sizeof(int));
  if (e == cudaSuccess) {
    d_sum = reinterpret_cast<int*>(d_act + nb);
    std::vector<int*> ha(nb);
    for (int b = 0; b < nb; ++b) ha[b] = gs[b]->S.active;
    e = cudaMemcpy(d_act, ha.data(), (size_t)nb * sizeof(int*), cudaMemcpyHostToDevice);
  }
  for (int b = 0; b <= nb && e == cudaSuccess; ++b) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    evs.push_back(ev);
  }
  // branch b's WHILE node at the capture point of its stream, its body captured on stw
  auto while_branch = [&](PGGraph<T>* g) -> cudaError_t {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e_ = cudaStreamGetCaptureInfo(g->st, &cs, nullptr, &cg, &deps, &ndeps);
    cudaGraphConditionalHandle hw = 0;
    if (e_ == cudaSuccess) e_ = cudaGraphConditionalHandleCreate(&hw, cg, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = hw;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wnode = nullptr;
    if (e_ == cudaSuccess) e_ = cudaGraphAddNode(&wnode, cg, deps, ndeps, &cp);
    if (e_ == cudaSuccess) e_ = cudaStreamUpdateCaptureDependencies(g->st, &wnode, 1, cudaStreamSetCaptureDependencies);
    if (e_ == cudaSuccess)
      e_ = cudaStreamBeginCaptureToGraph(g->stw, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal);
    if (e_ != cudaSuccess) return e_;
    cudaStream_t outer = g->st;
    g->st = g->stw;  // the body's kernels and IF nodes go into the WHILE body
    const int brc = g->capture(hw);
    g->st = outer;
    cudaGraph_t body = nullptr;
    e_ = cudaStreamEndCapture(g->stw, &body);
    if (brc && e_ == cudaSuccess) e_ = cudaErrorUnknown;
    return e_;
  };
  if (e == cudaSuccess) {
    e = cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(evs[nb], root);
    for (int b = 0; b < nb && e == cudaSuccess && !rc; ++b) {
      e = cudaStreamWaitEvent(gs[b]->st, evs[nb], 0);
      if (e == cudaSuccess) {
        if (loops) e = while_branch(gs[b]);
        else rc = gs[b]->capture();
      }
      if (e == cudaSuccess && !rc) e = cudaEventRecord(evs[b], gs[b]->st);
      if (e == cudaSuccess && !rc) e = cudaStreamWaitEvent(root, evs[b], 0);
    }
    if (e == cudaSuccess && !rc) {
      k_pg_sum_active<<<1, 32, 0, root>>>(d_act, nb, d_sum);
      note_launch();
    }
    const cudaError_t e2 = cudaStreamEndCapture(root, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&exec, graph, 0);
  }
  if (e != cudaSuccess && !rc) { set_cuda_error("graph solve capture", e); rc = 1; }
  long long launches = 0;
  if (!rc) {
    int cap = 0;
    for (auto* g : gs) cap = std::max(cap, g->io->maxit);
    // one launch per Krylov step (one target) or per whole solve (WHILE branches)
    const long long lim = loops ? 4 : (long long)cap + 64;
    const int per_poll = loops ? 1 : 4;
    while (e == cudaSuccess && launches < lim) {
      for (int k = 0; k < per_poll && e == cudaSuccess; ++k, ++launches) e = cudaGraphLaunch(exec, root);
      if (e == cudaSuccess) e = cudaMemcpyAsync(h_sum, d_sum, sizeof(int), cudaMemcpyDeviceToHost, root);
      if (e == cudaSuccess) e = cudaStreamSynchronize(root);
      if (e != cudaSuccess || *h_sum == 0) break;
    }
    if (e != cudaSuccess) { set_cuda_error("graph solve", e); rc = 1; }
    note_launch((unsigned long long)launches);  // the summing kernel
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (root) { cudaStreamSynchronize(root); cudaStreamDestroy(root); }
  for (auto ev : evs)
    if (ev) cudaEventDestroy(ev);
  cudaFree(d_act);
  cudaFreeHost(h_sum);
  return rc;
}

// Targets of a multi-target solve hand their graph iterations to one
// coordinator, which runs all of them as branches of one graph (pg_run).  Each
// target's solve calls join() at the hand-over point and blocks until the
// combined run ends; a target that finishes or fails without handing over calls
// leave().  run() (the coordinator's thread) waits until every target has done
// one of the two.
template <typename T> struct PGGroup {
  std::mutex m;
  std::condition_variable cv;
  int expected = 0, arrived = 0;
  bool done = false;
  int rc = 0;
  std::vector<PGGraph<T>*> graphs;
  int join(PGGraph<T>* g) {
    std::unique_lock<std::mutex> lk(m);
    graphs.push_back(g);
    ++arrived;
    cv.notify_all();
    cv.wait(lk, [&] { return done; });
    return rc;
  }
  void leave() {
    std::lock_guard<std::mutex> lk(m);
    ++arrived;
    cv.notify_all();
  }
  int run() {
    std::unique_lock<std::mutex> lk(m);
    cv.wait(lk, [&] { return arrived >= expected; });
    rc = pg_run<T>(graphs);
    done = true;
    cv.notify_all();
    return rc;
  }
};

template <typename T>
static int pbcgs2_graph_loop(BatchIO<T>& io, BatchOps<T>& ops, std::vector<int>& nc, cplx<T>* const* w, PGHost& hs,
                             double mv_ms_per_rhs) {
  PGGraph<T> g;
  int rc = g.init(io, ops, nc, w, hs, mv_ms_per_rhs);
  if (!rc) {
    PGGroup<T>* grp = static_cast<PGGroup<T>*>(io.group);
    if (grp) {
      io.group_joined = 1;
      rc = grp->join(&g);
    } else {
      rc = pg_run<T>({&g});
    }
  } else if (io.group) {
    io.group_joined = 1;
    static_cast<PGGroup<T>*>(io.group)->leave();
  }
  if (!rc) rc = g.readback();
  g.release();
  return rc;
}

// --------------------------------------------------------------------------
// PBCGS2 (per RHS: solvers.cu solve_pbcgs2, reference cu:459-480, cu:1168-1278)
template <typename T> int solve_batch_pbcgs2(BatchIO<T>& io, BatchResult& res) {
  using C = cplx<T>;
  BCtx<T> c(io);
  BatchOps<T>& ops = c.ops;
  const int R = io.R;
  C *rr = c.w(0), *r[3] = {c.w(1), c.w(2), c.w(3)}, *u[3] = {c.w(4), c.w(5), c.w(6)};
  C *XP = c.w(7), *BP = c.w(8), *X = c.w(9), *sy = c.w(10);
  const std::vector<double2> one = BCtx<T>::cst(R, 1.0), mone = BCtx<T>::cst(R, -1.0);
  res.itno.assign(R, 0); res.ncompte.assign(R, 0); res.status.assign(R, 0); res.tole.assign(R, 0.0);
  std::vector<int> live(R, 1);
  const int* MA = ops.mask(live);
  ops.copy(XP, io.x, MA);
  ops.copy(rr, io.b, MA); ops.copy(r[0], io.b, MA); ops.copy(BP, io.b, MA);
  for (C* v : {r[1], r[2], u[0], u[1], u[2], X}) ops.zero(v, MA);
  std::vector<double2> o;
  {
    const C* A1[1] = {r[0]};
    const int c1[1] = {1};
    if (ops.dots(1, A1, A1, c1, MA, o)) return 1;
  }
  std::vector<double> rnrm0(R), rnrm(R), mxx(R), mxr(R), resid(R);
  std::vector<Z> alpha(R, 0.0), omega(R, 1.0), sigma(R, 1.0), rho0(R, 1.0), rho1(R, 0.0), beta(R, 0.0);
  for (int i = 0; i < R; ++i) {
    rnrm0[i] = std::sqrt(std::max(0.0, o[i].x));
    rnrm[i] = mxx[i] = mxr[i] = rnrm0[i];
    resid[i] = rnrm0[i] > 0.0 ? 1.0 : 0.0;
  }
  std::vector<int> it(R, 0);
  int rc;
  // DDSCAT_B200_GRAPH with residual replacement: the first iteration runs
  // host-driven (it sizes the workspace and times the MATVEC), the rest as a
  // captured graph per iteration
  const bool use_graph = io.graph && io.replace;
  int host_iters = 0;
  for (;;) {
    std::vector<int> I(R, 0);
    for (int i = 0; i < R; ++i) I[i] = live[i] && resid[i] > io.tol && it[i] < io.maxit;
    if (!any_of(I)) break;
    if (use_graph && host_iters >= 1) {
      float t = 0.f;
      cudaStreamSynchronize(ops.stream);
      if (!c.ev.empty()) cudaEventElapsedTime(&t, c.ev.back().first, c.ev.back().second);
      const double per_rhs = c.last_cnt > 0 ? (double)t / c.last_cnt : 0.0;
      PGHost hs{alpha, omega, sigma, rho0, rho1, beta, rnrm0, rnrm, mxx, mxr, resid, it, live, res.status};
      C* wv[11] = {rr, r[0], r[1], r[2], u[0], u[1], u[2], XP, BP, X, sy};
      if ((rc = pbcgs2_graph_loop<T>(io, ops, c.nc, wv, hs, per_rhs))) return rc;
      resid = hs.resid;
      it = hs.it;
      live = hs.live;
      res.status = hs.status;
      break;
    }
    ++host_iters;
    for (int i = 0; i < R; ++i)
      if (I[i]) { it[i]++; rho0[i] = -(omega[i] * rho0[i]); }
    const int* MI = ops.mask(I);
    for (int k = 1; k <= 2; ++k) {
      {
        const C* A1[1] = {rr};
        const C* B1[1] = {r[k - 1]};
        const int c1[1] = {1};
        if (ops.dots(1, A1, B1, c1, MI, o)) return 1;
      }
      std::vector<double2> cb(R), ca(R), cma(R);
      for (int i = 0; i < R; ++i) {
        if (!I[i]) continue;
        rho1[i] = zd2(o[i]);
        if (rho0[i] == Z(0.0)) { res.status[i] = 95; live[i] = 0; I[i] = 0; continue; }
        beta[i] = alpha[i] * (rho1[i] / rho0[i]);
        rho0[i] = rho1[i];
        cb[i] = dz(-beta[i]);
      }
      MI = ops.mask(I);
      for (int j = 0; j < k; ++j) ops.lin(u[j], cb.data(), r[j], one.data(), nullptr, nullptr, MI);
      if ((rc = c.mv(u[k - 1], u[k], I))) return rc;
      {
        const C* A1[1] = {rr};
        const C* B1[1] = {u[k]};
        const int c1[1] = {1};
        if (ops.dots(1, A1, B1, c1, MI, o)) return 1;
      }
      for (int i = 0; i < R; ++i) {
        if (!I[i]) continue;
        sigma[i] = zd2(o[i]);
        if (sigma[i] == Z(0.0)) { res.status[i] = 98; live[i] = 0; I[i] = 0; continue; }
        alpha[i] = rho1[i] / sigma[i];
        ca[i] = dz(alpha[i]);
        cma[i] = dz(-alpha[i]);
      }
      MI = ops.mask(I);
      ops.lin(X, one.data(), u[0], ca.data(), nullptr, nullptr, MI);
      for (int j = 0; j < k; ++j) ops.lin(r[j], one.data(), u[j + 1], cma.data(), nullptr, nullptr, MI);
      if ((rc = c.mv(r[k - 1], r[k], I))) return rc;
      {
        const C* A1[1] = {r[0]};
        const int c1[1] = {1};
        if (ops.dots(1, A1, A1, c1, MI, o)) return 1;
      }
      for (int i = 0; i < R; ++i) {
        if (!I[i]) continue;
        rnrm[i] = std::sqrt(std::max(0.0, o[i].x));
        mxx[i] = std::max(mxx[i], rnrm[i]);
        mxr[i] = std::max(mxr[i], rnrm[i]);
      }
    }
    {
      const C* A6[6] = {r[0], r[1], r[1], r[2], r[2], r[2]};
      const C* B6[6] = {r[0], r[0], r[1], r[0], r[1], r[2]};
      const int c6[6] = {1, 1, 1, 1, 1, 1};
      if (ops.dots(6, A6, B6, c6, MI, o)) return 1;
    }
    std::vector<double2> cy1(R), cy2(R), cmy1(R), cmy2(R);
    std::vector<int> XPDT(R, 0), RCMP(R, 0);
    for (int i = 0; i < R; ++i) {
      if (!I[i]) continue;
      Z Zm[3][3];
      Zm[0][0] = zd2(o[6 * i]); Zm[1][0] = zd2(o[6 * i + 1]); Zm[1][1] = zd2(o[6 * i + 2]);
      Zm[2][0] = zd2(o[6 * i + 3]); Zm[2][1] = zd2(o[6 * i + 4]); Zm[2][2] = zd2(o[6 * i + 5]);
      Zm[0][1] = std::conj(Zm[1][0]); Zm[0][2] = std::conj(Zm[2][0]); Zm[1][2] = std::conj(Zm[2][1]);
      auto matv = [&](const Z* v, Z* out) {
        for (int a = 0; a < 3; ++a) { out[a] = 0.0; for (int b = 0; b < 3; ++b) out[a] += Zm[a][b] * v[b]; }
      };
      auto inner = [](const Z* a, const Z* b) { Z sum = 0.0; for (int k = 0; k < 3; ++k) sum += std::conj(a[k]) * b[k]; return sum; };
      if (Zm[1][1] == Z(0.0)) { res.status[i] = 102; live[i] = 0; I[i] = 0; continue; }
      Z y0[3] = {-1.0, Zm[1][0] / Zm[1][1], 0.0}, yl[3] = {0.0, Zm[1][2] / Zm[1][1], -1.0}, zy0[3], zyl[3];
      matv(y0, zy0);
      matv(yl, zyl);
      const double k0 = std::sqrt(std::abs(inner(y0, zy0))), kl = std::sqrt(std::abs(inner(yl, zyl)));
      if (k0 == 0.0 || kl == 0.0) { res.status[i] = 102; live[i] = 0; I[i] = 0; continue; }
      const Z vr = inner(yl, zy0) / (k0 * kl);
      const double avr = std::abs(vr);
      if (avr == 0.0) { res.status[i] = 102; live[i] = 0; I[i] = 0; continue; }
      const Z fac = vr * (std::max(avr, 0.7) / avr) * (k0 / kl);
      for (int a = 0; a < 3; ++a) y0[a] -= fac * yl[a];
      omega[i] = y0[2];
      matv(y0, zy0);
      rnrm[i] = std::sqrt(std::abs(inner(y0, zy0)));
      mxx[i] = std::max(mxx[i], rnrm[i]);
      mxr[i] = std::max(mxr[i], rnrm[i]);
      cy1[i] = dz(y0[1]); cy2[i] = dz(y0[2]); cmy1[i] = dz(-y0[1]); cmy2[i] = dz(-y0[2]);
      XPDT[i] = rnrm[i] < 1.0e-2 * rnrm0[i] && rnrm0[i] < mxx[i];
      RCMP[i] = (rnrm[i] < 1.0e-2 * mxr[i] && rnrm0[i] < mxr[i]) || XPDT[i];
      resid[i] = rnrm0[i] > 0.0 ? rnrm[i] / rnrm0[i] : 0.0;
    }
    MI = ops.mask(I);
    ops.lin(u[0], one.data(), u[1], cmy1.data(), u[2], cmy2.data(), MI);
    ops.lin(X, one.data(), r[0], cy1.data(), r[1], cy2.data(), MI);
    ops.lin(r[0], one.data(), r[1], cmy1.data(), r[2], cmy2.data(), MI);
    std::vector<int> CK(R, 0), RS(R, 0), RP(R, 0);
    for (int i = 0; i < R; ++i) CK[i] = I[i] && ((it[i] % 20) == 0 || resid[i] <= io.tol);
    if (any_of(CK)) {
      if ((rc = c.mv(X, sy, CK))) return rc;
      std::vector<double2> nn;
      if (ops.diff_norms(BP, sy, r[0], ops.mask(CK), nn)) return 1;
      for (int i = 0; i < R; ++i) {
        if (!CK[i]) continue;
        const double tr = std::sqrt(std::max(0.0, nn[2 * i].x)), gapn = std::sqrt(std::max(0.0, nn[2 * i + 1].x));
        const double tres = tr / rnrm0[i];
        const double gap = tr > 0.0 ? gapn / tr : (gapn == 0.0 ? 0.0 : INFINITY);
        const bool conv = tres <= io.tol;
        const bool rest = gap >= 1.0e-3 || (resid[i] <= io.tol && !conv);
        if (conv) { resid[i] = tres; live[i] = 0; I[i] = 0; continue; }
        if (rest && io.replace) { RP[i] = 1; resid[i] = tres; }
        else if (rest) { RS[i] = 1; resid[i] = tres; I[i] = 0; }
      }
      if (any_of(RP)) {
        // residual replacement: r0 = BP - A X, shadow residual and search
        // directions kept
        ops.lin(r[0], nullptr, BP, one.data(), sy, mone.data(), ops.mask(RP));
        for (int i = 0; i < R; ++i)
          if (RP[i]) { rnrm[i] = resid[i] * rnrm0[i]; mxr[i] = std::max(mxr[i], rnrm[i]); }
      }
      if (any_of(RS)) {
        const int* MR = ops.mask(RS);
        // r0 = BP - A X  (sy holds A X)
        ops.lin(r[0], nullptr, BP, one.data(), sy, mone.data(), MR);
        ops.lin(XP, one.data(), X, one.data(), nullptr, nullptr, MR);
        ops.zero(X, MR);
        ops.copy(BP, r[0], MR);
        ops.copy(rr, r[0], MR);
        for (C* v : {r[1], r[2], u[0], u[1], u[2]}) ops.zero(v, MR);
        for (int i = 0; i < R; ++i)
          if (RS[i]) {
            rnrm[i] = mxx[i] = mxr[i] = resid[i] * rnrm0[i];
            alpha[i] = 0.0; omega[i] = 1.0; sigma[i] = 1.0; rho0[i] = 1.0;
          }
      }
    }
    std::vector<int> RC(R, 0), XD(R, 0);
    for (int i = 0; i < R; ++i) { RC[i] = I[i] && RCMP[i]; XD[i] = RC[i] && XPDT[i]; }
    if (any_of(RC)) {
      if ((rc = c.mv(X, sy, RC))) return rc;
      const int* MC = ops.mask(RC);
      ops.lin(r[0], nullptr, BP, one.data(), sy, mone.data(), MC);
      if (any_of(XD)) {
        const int* MX = ops.mask(XD);
        ops.lin(XP, one.data(), X, one.data(), nullptr, nullptr, MX);
        ops.zero(X, MX);
        ops.copy(BP, r[0], MX);
      }
      for (int i = 0; i < R; ++i)
        if (RC[i]) { mxr[i] = rnrm[i]; if (XD[i]) mxx[i] = rnrm[i]; }
    }
  }
  // X += XP and one final true residual against b (cu:1259-1264)
  std::vector<int> F(R, 0);
  for (int i = 0; i < R; ++i) F[i] = res.status[i] == 0;
  const int* MF = ops.mask(F);
  ops.lin(X, one.data(), XP, one.data(), nullptr, nullptr, MF);
  if ((rc = c.mv(X, sy, F))) return rc;
  std::vector<double2> nn;
  if (ops.diff_norms(io.b, sy, io.b, MF, nn)) return 1;
  ops.copy(io.x, X, MF);
  c.finish_timing();
  for (int i = 0; i < R; ++i) {
    res.itno[i] = it[i];
    res.ncompte[i] = c.nc[i];
    res.tole[i] = F[i] ? (rnrm0[i] > 0.0 ? std::sqrt(std::max(0.0, nn[2 * i].x)) / rnrm0[i] : INFINITY) : resid[i];
  }
  return 0;
}

template struct BatchOps<float>;
template struct BatchOps<double>;
template int solve_batch_qmrccg<float>(BatchIO<float>&, BatchResult&);
template int solve_batch_qmrccg<double>(BatchIO<double>&, BatchResult&);
template int solve_batch_pbcgs2<float>(BatchIO<float>&, BatchResult&);
template int solve_batch_pbcgs2<double>(BatchIO<double>&, BatchResult&);

void* pg_group_create(int expected) {
  auto* g = new PGGroup<float>();
  g->expected = expected;
  return g;
}
int pg_group_run(void* grp) { return static_cast<PGGroup<float>*>(grp)->run(); }
void pg_group_leave(void* grp) { static_cast<PGGroup<float>*>(grp)->leave(); }
void pg_group_destroy(void* grp) { delete static_cast<PGGroup<float>*>(grp); }

}  // namespace ddb
