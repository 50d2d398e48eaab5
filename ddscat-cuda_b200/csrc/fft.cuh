// Self-written mixed-radix complex FFT building blocks (sm_100a).
//
// Algorithm: the self-sorting Stockham formulation of Govindaraju et al.,
// "High Performance Discrete Fourier Transforms on Graphics Processors"
// (SC 2008): stage with radix R and running product Ns reads
// src[j + r*N/R], twiddles by exp(dir*2*pi*i*r*(j%Ns)/(Ns*R)), applies an
// R-point DFT and writes dst[(j/Ns)*Ns*R + j%Ns + r*Ns].  Stages ping-pong
// between two shared-memory tiles; radices 2,3,4,5,8 have hand-written
// butterflies and any other prime uses an O(R^2) butterfly from the twiddle
// table, so every transform length the DDSCAT grid can produce is handled.
//
// The transforms here replace the cuFFT C2C plans of the reference
// (ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu:410, :412, :649, :674).
// Convention: dir = +1 is exp(+i...) (the reference's CUFFT_INVERSE, used
// first on the padded polarisation and for the Green tensor), dir = -1 is
// exp(-i...), both unnormalised.
#pragma once
#include "common.cuh"

namespace ddb {

constexpr int FFT_MAX_STAGES = 16;

struct FftPlan {
  int n = 0;
  int nstages = 0;
  int radix[FFT_MAX_STAGES] = {0};
};

// Host: factor n into radices, 8 first (fewest passes), then 4, 2, 3, 5 and
// any remaining primes.
inline FftPlan make_fft_plan(int n) {
  FftPlan p;
  p.n = n;
  int m = n;
  const int pref[5] = {8, 4, 2, 3, 5};
  for (int t = 0; t < 5; ++t)
    while (m % pref[t] == 0 && p.nstages < FFT_MAX_STAGES) { p.radix[p.nstages++] = pref[t]; m /= pref[t]; }
  for (int q = 7; m > 1 && p.nstages < FFT_MAX_STAGES; q += 2)
    while (m % q == 0 && p.nstages < FFT_MAX_STAGES) { p.radix[p.nstages++] = q; m /= q; }
  if (m != 1) p.nstages = -1;  // unsupported (too many stages)
  return p;
}

// ---- butterflies: in-register R-point DFTs, W = exp(dir*2*pi*i/R) ---------
template <int DIR, typename C> __device__ __forceinline__ void bfly2(C* v) {
  C a = v[0], b = v[1];
  v[0] = vadd(a, b);
  v[1] = vsub(a, b);
}
template <int DIR, typename C> __device__ __forceinline__ void bfly4(C* v) {
  const C s02 = vadd(v[0], v[2]), d02 = vsub(v[0], v[2]);
  const C s13 = vadd(v[1], v[3]), t13 = vsub(v[1], v[3]);
  v[0] = vadd(s02, s13);
  v[2] = vsub(s02, s13);
  v[1] = addrot<DIR>(d02, t13);  // d02 + DIR*i*t13
  v[3] = subrot<DIR>(d02, t13);
}
// W8^1 * o and W8^3 * o, W8 = exp(DIR*2*pi*i/8) = (1 + DIR*i)/sqrt2
template <int DIR, typename C> __device__ __forceinline__ C w8_1(C o) {
  using R = decltype(o.x);
  const R h = (R)0.70710678118654752440;
  return DIR > 0 ? mk2<C>(h * (o.x - o.y), h * (o.y + o.x)) : mk2<C>(h * (o.x + o.y), h * (o.y - o.x));
}
template <int DIR, typename C> __device__ __forceinline__ C w8_3(C o) {
  using R = decltype(o.x);
  const R h = (R)0.70710678118654752440, hn = (R)-0.70710678118654752440;
  return DIR > 0 ? mk2<C>(hn * (o.x + o.y), h * (o.x - o.y)) : mk2<C>(h * (o.y - o.x), hn * (o.x + o.y));
}
// DIR*i*o
template <int DIR, typename C> __device__ __forceinline__ C rot4(C o) {
  using R = decltype(o.x);
  const R m1 = (R)-1.0;
  return DIR > 0 ? mk2<C>(m1 * o.y, o.x) : mk2<C>(o.y, m1 * o.x);
}
template <int DIR, typename C> __device__ __forceinline__ void bfly8(C* v) {
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  bfly4<DIR>(e);
  bfly4<DIR>(o);
  const C t1 = w8_1<DIR>(o[1]), t3 = w8_3<DIR>(o[3]);
  v[0] = vadd(e[0], o[0]);
  v[4] = vsub(e[0], o[0]);
  v[1] = vadd(e[1], t1);
  v[5] = vsub(e[1], t1);
  v[2] = addrot<DIR>(e[2], o[2]);  // e2 + W8^2 o2, W8^2 = DIR*i
  v[6] = subrot<DIR>(e[2], o[2]);
  v[3] = vadd(e[3], t3);
  v[7] = vsub(e[3], t3);
}
template <int DIR, typename C> __device__ __forceinline__ void bfly3(C* v) {
  using R = decltype(v[0].x);
  const R c = (R)-0.5, s = (R)(DIR * 0.86602540378443864676), ms = (R)(-DIR * 0.86602540378443864676);
  const C t = vadd(v[1], v[2]);
  const C d = vsub(v[1], v[2]);
  const C a = v[0];
  const C m = mk2<C>(a.x + c * t.x, a.y + c * t.y);
  const C u = mk2<C>(ms * d.y, s * d.x);
  v[0] = vadd(a, t);
  v[1] = vadd(m, u);
  v[2] = vsub(m, u);
}
template <int DIR, typename C> __device__ __forceinline__ void bfly5(C* v) {
  using R = decltype(v[0].x);
  const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
  const R s1 = (R)(DIR * 0.95105651629515357212), s2 = (R)(DIR * 0.58778525229247312917);
  C a = v[0];
  C t1 = cadd(v[1], v[4]), d1 = csub(v[1], v[4]);
  C t2 = cadd(v[2], v[3]), d2 = csub(v[2], v[3]);
  C m1 = mk<C>((double)(a.x + c1 * t1.x + c2 * t2.x), (double)(a.y + c1 * t1.y + c2 * t2.y));
  C m2 = mk<C>((double)(a.x + c2 * t1.x + c1 * t2.x), (double)(a.y + c2 * t1.y + c1 * t2.y));
  // i*(s1 d1 + s2 d2) and i*(s2 d1 - s1 d2)
  C u1 = mk<C>((double)(-(s1 * d1.y + s2 * d2.y)), (double)(s1 * d1.x + s2 * d2.x));
  C u2 = mk<C>((double)(-(s2 * d1.y - s1 * d2.y)), (double)(s2 * d1.x - s1 * d2.x));
  v[0] = cadd(a, cadd(t1, t2));
  v[1] = cadd(m1, u1);
  v[4] = csub(m1, u1);
  v[2] = cadd(m2, u2);
  v[3] = csub(m2, u2);
}

template <int R, int DIR, typename C> __device__ __forceinline__ void bfly(C* v) {
  if constexpr (R == 2) bfly2<DIR>(v);
  else if constexpr (R == 3) bfly3<DIR>(v);
  else if constexpr (R == 4) bfly4<DIR>(v);
  else if constexpr (R == 5) bfly5<DIR>(v);
  else if constexpr (R == 8) bfly8<DIR>(v);
}

// twiddle exp(dir*2*pi*i*m/N) from the table tw[m] = exp(-2*pi*i*m/N)
template <int DIR, typename C> __device__ __forceinline__ C twid(const C* __restrict__ tw, int m) {
  C w = tw[m];
  if (DIR > 0) w.y = -w.y;
  return w;
}

// Tile addressing: element e of line l lives at l*ls + e*es.
struct Lay {
  int ls, es;
  __device__ __forceinline__ int at(int l, int e) const { return l * ls + e * es; }
};

template <int R, int DIR, typename C>
__device__ __forceinline__ void stage_fixed(const C* __restrict__ src, C* __restrict__ dst, Lay lay, int nlines, int N,
                                            int Ns, const C* __restrict__ tw) {
  const int NR = N / R;
  const int items = nlines * NR;
  const int tstep = N / (Ns * R);
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int l = it % nlines;
    const int j = it / nlines;
    const int k = j % Ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[lay.at(l, j + r * NR)];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], twid<DIR>(tw, (r * k * tstep) % N));
    }
    bfly<R, DIR>(v);
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[lay.at(l, idxD + r * Ns)] = v[r];
  }
}

// Generic prime radix: O(R^2) with W_R^{rq} = tw[(r*q mod R) * N/R].
template <int DIR, typename C>
__device__ void stage_generic(const C* __restrict__ src, C* __restrict__ dst, Lay lay, int nlines, int N, int Ns, int R,
                              const C* __restrict__ tw) {
  const int NR = N / R;
  const int items = nlines * NR;
  const int tstep = N / (Ns * R);
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int l = it % nlines;
    const int j = it / nlines;
    const int k = j % Ns;
    const int idxD = (j / Ns) * Ns * R + k;
    for (int q = 0; q < R; ++q) {
      double2 acc = make_double2(0.0, 0.0);
      for (int r = 0; r < R; ++r) {
        C v = src[lay.at(l, j + r * NR)];
        if (Ns > 1 && r > 0) v = cmul(v, twid<DIR>(tw, (r * k * tstep) % N));
        C w = twid<DIR>(tw, ((r * q) % R) * NR);
        C p = cmul(v, w);
        acc.x += (double)p.x;
        acc.y += (double)p.y;
      }
      dst[lay.at(l, idxD + q * Ns)] = from_d<C>(acc);
    }
  }
}

// Full transform of `nlines` lines held in tile A (scratch tile B of the same
// shape).  Returns the tile that holds the result.  Must be called by the
// whole block; ends with a barrier.
template <int DIR, typename C>
__device__ C* fft_tile(C* A, C* B, Lay lay, int nlines, const FftPlan& p, const C* __restrict__ tw) {
  C* src = A;
  C* dst = B;
  int Ns = 1;
  const int N = p.n;
  for (int s = 0; s < p.nstages; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 2: stage_fixed<2, DIR>(src, dst, lay, nlines, N, Ns, tw); break;
      case 3: stage_fixed<3, DIR>(src, dst, lay, nlines, N, Ns, tw); break;
      case 4: stage_fixed<4, DIR>(src, dst, lay, nlines, N, Ns, tw); break;
      case 5: stage_fixed<5, DIR>(src, dst, lay, nlines, N, Ns, tw); break;
      case 8: stage_fixed<8, DIR>(src, dst, lay, nlines, N, Ns, tw); break;
      default: stage_generic<DIR>(src, dst, lay, nlines, N, Ns, R, tw); break;
    }
    __syncthreads();
    C* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

}  // namespace ddb
