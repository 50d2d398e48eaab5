// Krylov vector kernels and FP64 inner products (sm_100a).
//
// Replaces the reference's chunked convert-to-complex-double + cublasZdotc /
// cublasZdotu / cublasDznrm2 path and its CPU accumulation of chunk partials
// (ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu:224-335): each product is one
// pass that loads the FP32 vectors, accumulates in FP64 (warp shuffles, then a
// block tree), writes one partial per block, and the last block to finish sums
// the partials in a fixed order, so results are deterministic and no host
// round trip is needed to combine chunks.
#include <algorithm>
#include "engine.h"

namespace ddb {

constexpr int RED_THREADS = 256;
constexpr int RED_MAXK = 8;

template <typename T> struct DotSpec {
  const cplx<T>* a[RED_MAXK];
  const cplx<T>* b[RED_MAXK];
  const cplx<T>* c[RED_MAXK];
  int conj[RED_MAXK];
  int mode;  // 0: sum op(a)*b ; 1: sum |a-b|^2 ; 2: sum |a-b-c|^2
  int k;
};

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// KM: the largest product count of the launch (registers scale with it)
template <typename T, int KM>
__global__ void __launch_bounds__(RED_THREADS) k_dots(int n, DotSpec<T> sp, double2* partials, double2* out,
                                                      unsigned* count) {
  __shared__ double2 wsum[RED_MAXK][RED_THREADS / 32];
  __shared__ bool last;
  double2 acc[KM];
#pragma unroll
  for (int q = 0; q < KM; ++q) acc[q] = make_double2(0.0, 0.0);
  // two elements per thread and round, all of a round's loads issued before
  // its products, so that a thread keeps several loads in flight
  auto term = [&](int q, const cplx<T>& av, const cplx<T>& bv, const cplx<T>* cp, int i) {
    const double2 a = to_d(av), b = to_d(bv);
    if (sp.mode == 0) {
      if (sp.conj[q]) {
        acc[q].x += a.x * b.x + a.y * b.y;
        acc[q].y += a.x * b.y - a.y * b.x;
      } else {
        acc[q].x += a.x * b.x - a.y * b.y;
        acc[q].y += a.x * b.y + a.y * b.x;
      }
    } else {
      double dr = a.x - b.x, di = a.y - b.y;
      if (sp.mode == 2) {
        const double2 c = to_d(cp[i]);
        dr -= c.x;
        di -= c.y;
      }
      acc[q].x += dr * dr + di * di;
    }
  };
  const int stride = gridDim.x * blockDim.x;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + stride < n; i += 2 * stride) {
    cplx<T> a0[KM], b0[KM], a1[KM], b1[KM];
#pragma unroll
    for (int q = 0; q < KM; ++q) {
      if (q >= sp.k) break;
      a0[q] = sp.a[q][i]; b0[q] = sp.b[q][i];
      a1[q] = sp.a[q][i + stride]; b1[q] = sp.b[q][i + stride];
    }
#pragma unroll
    for (int q = 0; q < KM; ++q) {
      if (q >= sp.k) break;
      term(q, a0[q], b0[q], sp.c[q], i);
      term(q, a1[q], b1[q], sp.c[q], i + stride);
    }
  }
  if (i < n) {
#pragma unroll
    for (int q = 0; q < KM; ++q) {
      if (q >= sp.k) break;
      term(q, sp.a[q][i], sp.b[q][i], sp.c[q], i);
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < KM; ++q) {  // compile-time indices: acc stays in registers
    if (q >= sp.k) break;
    double2 v = warp_sum(acc[q]);
    if (lane == 0) wsum[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int q = 0; q < sp.k; ++q) {
      double2 v = (lane < RED_THREADS / 32) ? wsum[q][lane] : make_double2(0.0, 0.0);
      v = warp_sum(v);
      if (lane == 0) partials[(size_t)q * gridDim.x + blockIdx.x] = v;
    }
  }
  __threadfence();
  if (threadIdx.x == 0) last = (atomicInc(count, gridDim.x - 1) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the last block sums the partials in block order (deterministic)
  for (int q = 0; q < sp.k; ++q) {
    double2 v = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
      const volatile double* pp = reinterpret_cast<volatile double*>(partials + (size_t)q * gridDim.x + b);
      v.x += pp[0];
      v.y += pp[1];
    }
    v = warp_sum(v);
    if (lane == 0) wsum[q][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int q = 0; q < sp.k; ++q) {
      double2 v = (lane < RED_THREADS / 32) ? wsum[q][lane] : make_double2(0.0, 0.0);
      v = warp_sum(v);
      if (lane == 0) out[q] = v;
    }
  }
}

template <typename T> int VecOps<T>::init(cudaStream_t s) {
  stream = s;
  nblocks = 8 * 148;  // capacity of the partials buffer; launch_dots sizes each launch to one resident wave
  cudaError_t e = cudaMalloc((void**)&d_red, (size_t)RED_MAXK * nblocks * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_out, RED_MAXK * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_count, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMallocHost((void**)&h_out, RED_MAXK * sizeof(double2));
  if (e != cudaSuccess) { set_cuda_error("reduction buffers", e); return 1; }
  cudaMemset(d_count, 0, sizeof(unsigned));
  return 0;
}

template <typename T> void VecOps<T>::release() {
  cudaFree(d_red); cudaFree(d_out); cudaFree(d_count);
  if (h_out) cudaFreeHost(h_out);
  d_red = d_out = nullptr; d_count = nullptr; h_out = nullptr;
}

// One launch of KM-product blocks, as many as are resident at once (the
// register count grows with KM; nb caps them at the partials buffer), so the
// grid-stride loop runs in a single wave.
template <typename T>
static void launch_dots(int nb, cudaStream_t st, int n, DotSpec<T>& sp, double2* red, double2* out, unsigned* cnt) {
  const int per_sm = sp.k <= 1 ? 8 : (sp.k <= 2 ? 6 : (sp.k <= 4 ? 3 : 2));
  nb = std::min(nb, 148 * per_sm);
  if (sp.k <= 1) k_dots<T, 1><<<nb, RED_THREADS, 0, st>>>(n, sp, red, out, cnt);
  else if (sp.k <= 2) k_dots<T, 2><<<nb, RED_THREADS, 0, st>>>(n, sp, red, out, cnt);
  else if (sp.k <= 4) k_dots<T, 4><<<nb, RED_THREADS, 0, st>>>(n, sp, red, out, cnt);
  else k_dots<T, RED_MAXK><<<nb, RED_THREADS, 0, st>>>(n, sp, red, out, cnt);
  note_launch();
}

template <typename T> static int run_dots(VecOps<T>& o, int n, DotSpec<T>& sp, double2* host_out) {
  int nb = o.nblocks;
  const int need = (int)ceil_div((size_t)std::max(n, 1), RED_THREADS);
  if (need < nb) nb = need;
  launch_dots<T>(nb, o.stream, n, sp, o.d_red, o.d_out, o.d_count);
  if (check_launch("FP64 inner product")) return 1;
  cudaError_t e = cudaMemcpyAsync(o.h_out, o.d_out, sp.k * sizeof(double2), cudaMemcpyDeviceToHost, o.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(o.stream);
  if (e != cudaSuccess) { set_cuda_error("inner product D2H", e); return 1; }
  for (int q = 0; q < sp.k; ++q) host_out[q] = o.h_out[q];
  return 0;
}

template <typename T>
int VecOps<T>::dots(int n, int k, const C* const* a, const C* const* b, const int* conjf, double2* host_out) {
  DotSpec<T> sp{};
  sp.k = k;
  sp.mode = 0;
  for (int q = 0; q < k; ++q) { sp.a[q] = a[q]; sp.b[q] = b[q]; sp.conj[q] = conjf[q]; }
  return run_dots(*this, n, sp, host_out);
}

template <typename T>
int VecOps<T>::dots_dev(int n, int k, const C* const* a, const C* const* b, const int* conjf) {
  DotSpec<T> sp{};
  sp.k = k;
  sp.mode = 0;
  for (int q = 0; q < k; ++q) { sp.a[q] = a[q]; sp.b[q] = b[q]; sp.conj[q] = conjf[q]; }
  int nb = nblocks;
  const int need = (int)ceil_div((size_t)std::max(n, 1), RED_THREADS);
  if (need < nb) nb = need;
  launch_dots<T>(nb, stream, n, sp, d_red, d_out, d_count);
  return check_launch("FP64 inner product");
}

template <typename T> double2 VecOps<T>::dotc(int n, const C* a, const C* b, int* err) {
  double2 r = make_double2(0, 0);
  const int cj = 1;
  if (dots(n, 1, &a, &b, &cj, &r)) *err = 1;
  return r;
}
template <typename T> double2 VecOps<T>::dotu(int n, const C* a, const C* b, int* err) {
  double2 r = make_double2(0, 0);
  const int cj = 0;
  if (dots(n, 1, &a, &b, &cj, &r)) *err = 1;
  return r;
}
template <typename T> double VecOps<T>::nrm2(int n, const C* a, int* err) {
  double v = dotc(n, a, a, err).x;
  if (v < 0.0 && v > -1e-12) v = 0.0;
  return std::sqrt(v > 0.0 ? v : 0.0);
}
template <typename T> double VecOps<T>::norm_diff(int n, const C* a, const C* b, int* err) {
  DotSpec<T> sp{};
  sp.k = 1; sp.mode = 1; sp.a[0] = a; sp.b[0] = b;
  double2 r;
  if (run_dots(*this, n, sp, &r)) { *err = 1; return 0.0; }
  return std::sqrt(std::max(0.0, r.x));
}
template <typename T> double VecOps<T>::norm_gap(int n, const C* a, const C* b, const C* c, int* err) {
  DotSpec<T> sp{};
  sp.k = 1; sp.mode = 2; sp.a[0] = a; sp.b[0] = b; sp.c[0] = c;
  double2 r;
  if (run_dots(*this, n, sp, &r)) { *err = 1; return 0.0; }
  return std::sqrt(std::max(0.0, r.x));
}

// ---------------------------------------------------------------- elementwise
template <typename C> __global__ void k_copy(C* d, const C* a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = a[i];
}
template <typename C> __global__ void k_zero(C* d, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = mk<C>(0, 0);
}
template <typename C> __global__ void k_diff(C* d, const C* a, const C* b, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = csub(a[i], b[i]);
}
template <typename C>
__global__ void k_lincomb(C* d, double2 zd, const C* a, double2 za, const C* b, double2 zb, int n) {
  const bool keep_d = !(zd.x == 0.0 && zd.y == 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    C v = mk<C>(0, 0);
    if (keep_d) v = (zd.x == 1.0 && zd.y == 0.0) ? d[i] : zmulv(zd, d[i]);
    if (a) v = cadd(v, (za.x == 1.0 && za.y == 0.0) ? a[i] : zmulv(za, a[i]));
    if (b) v = cadd(v, (zb.x == 1.0 && zb.y == 0.0) ? b[i] : zmulv(zb, b[i]));
    d[i] = v;
  }
}
template <typename C>
__global__ void k_precon(C* d, const C* a, const C* adia, const int* occ, int nat, int nat0) {
  const int n = 3 * nat0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i / nat0, k = i - c * nat0;
    const double2 q = zdiv(to_d(a[i]), to_d(adia[(size_t)c * nat + occ[k]]));
    d[i] = from_d<C>(q);
  }
}
template <typename C> __global__ void k_gather(const C* full, C* compact, const int* occ, int nat, int nat0) {
  const int n = 3 * nat0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i / nat0, k = i - c * nat0;
    compact[i] = full[(size_t)c * nat + occ[k]];
  }
}
template <typename C> __global__ void k_scatter(const C* compact, C* full, const int* occ, int nat, int nat0) {
  const int n = 3 * nat0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int c = i / nat0, k = i - c * nat0;
    full[(size_t)c * nat + occ[k]] = compact[i];
  }
}

static inline unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>(ceil_div(std::max<size_t>(n, 1), 256), 148 * 16); }

template <typename T> void v_copy(cplx<T>* d, const cplx<T>* a, int n, cudaStream_t s) {
  k_copy<<<grid_for(n), 256, 0, s>>>(d, a, n);
  note_launch();
}
template <typename T> void v_zero(cplx<T>* d, int n, cudaStream_t s) { k_zero<<<grid_for(n), 256, 0, s>>>(d, n); }
template <typename T> void v_diff(cplx<T>* d, const cplx<T>* a, const cplx<T>* b, int n, cudaStream_t s) {
  k_diff<<<grid_for(n), 256, 0, s>>>(d, a, b, n);
  note_launch();
}
template <typename T>
void v_lincomb(cplx<T>* d, double2 zd, const cplx<T>* a, double2 za, const cplx<T>* b, double2 zb, int n, cudaStream_t s) {
  k_lincomb<<<grid_for(n), 256, 0, s>>>(d, zd, a, za, b, zb, n);
  note_launch();
}
template <typename T>
void v_precon(cplx<T>* d, const cplx<T>* a, const cplx<T>* adia_full, const int* occ, int nat, int nat0, cudaStream_t s) {
  k_precon<<<grid_for((size_t)3 * nat0), 256, 0, s>>>(d, a, adia_full, occ, nat, nat0);
  note_launch();
}
template <typename T> void v_gather(const cplx<T>* full, cplx<T>* compact, const int* occ, int nat, int nat0, cudaStream_t s) {
  k_gather<<<grid_for((size_t)3 * nat0), 256, 0, s>>>(full, compact, occ, nat, nat0);
  note_launch();
}
template <typename T> void v_scatter(const cplx<T>* compact, cplx<T>* full, const int* occ, int nat, int nat0, cudaStream_t s) {
  k_scatter<<<grid_for((size_t)3 * nat0), 256, 0, s>>>(compact, full, occ, nat, nat0);
  note_launch();
}

#define DDB_INST(T)                                                                                              \
  template struct VecOps<T>;                                                                                     \
  template void v_copy<T>(cplx<T>*, const cplx<T>*, int, cudaStream_t);                                          \
  template void v_zero<T>(cplx<T>*, int, cudaStream_t);                                                          \
  template void v_diff<T>(cplx<T>*, const cplx<T>*, const cplx<T>*, int, cudaStream_t);                          \
  template void v_lincomb<T>(cplx<T>*, double2, const cplx<T>*, double2, const cplx<T>*, double2, int, cudaStream_t); \
  template void v_precon<T>(cplx<T>*, const cplx<T>*, const cplx<T>*, const int*, int, int, cudaStream_t);       \
  template void v_gather<T>(const cplx<T>*, cplx<T>*, const int*, int, int, cudaStream_t);                       \
  template void v_scatter<T>(const cplx<T>*, cplx<T>*, const int*, int, int, cudaStream_t);
DDB_INST(float)
DDB_INST(double)
#undef DDB_INST

}  // namespace ddb
