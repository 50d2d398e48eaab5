// Register-resident line FFT for power-of-two lengths N = E*T in {16..512}.
//
// A line is held by T threads, thread t owning elements t + T*i (i < E).  The
// transform is the four-step factorisation N = E*T: an E-point DFT in
// registers over i, a twiddle W_N^{t p}, one transpose through shared memory,
// and T-point DFTs in registers.  With E = m*T (m = 1 or 2) the output lands
// in the same index map (thread t owns X[t + T*i]), so a forward transform,
// a pointwise operation and an inverse transform chain without moving data,
// pad-skip loads read only i with t + T*i < n, and truncated stores write only
// the first n outputs.  In-register DFTs of 16 and 32 points are themselves
// four-step products of 4- and 8-point butterflies with exact constant
// twiddles.  Convention as in fft.cuh: DIR = +1 is exp(+i...), unnormalised.
#pragma once
#include "fft.cuh"

namespace ddb {

#include "w96.inc"

// W_K^m for DIR: exp(DIR * 2*pi*i*m/K), K divides 96
template <int K, int DIR, typename C> DDB_HD C wk(int m) {
  static_assert(96 % K == 0, "in-register DFT sizes must divide 96");
  const int q = (m * (96 / K)) % 96;
  return mk<C>(w96re(q), DIR < 0 ? w96im(q) : -w96im(q));
}

// x * W_K^m: the multiples of pi/4 are a rotation, a negation or the radix-8
// forms (m is a compile-time constant after unrolling, so the branches fold)
template <int K, int DIR, typename C> __device__ __forceinline__ C cmul_wk(C x, int m) {
  const int q = (m * (96 / K)) % 96;
  using R = decltype(x.x);
  const R m1 = (R)-1.0;
  if (q == 0) return x;
  if (q == 48) return mk2<C>(m1 * x.x, m1 * x.y);
  if (q == 24) return rot4<DIR>(x);
  if (q == 72) return rot4<-DIR>(x);
  if (q == 12) return w8_1<DIR>(x);
  if (q == 36) return w8_3<DIR>(x);
  if (q == 60) return w8_3<-DIR>(x);  // exp(5 i pi/4) = exp(-3 i pi/4)
  if (q == 84) return w8_1<-DIR>(x);  // exp(7 i pi/4) = exp(-i pi/4)
  return cmul(x, wk<K, DIR, C>(m));
}

// first factor of the four-step split K = K1 * K2 of an in-register DFT
template <int K> constexpr int dft_split() { return (K == 16 || K == 12) ? 4 : 8; }

template <int K, int DIR, typename C> __device__ __forceinline__ void dftr(C* v) {
  if constexpr (K == 1) {
  } else if constexpr (K == 2) {
    bfly2<DIR>(v);
  } else if constexpr (K == 4) {
    bfly4<DIR>(v);
  } else if constexpr (K == 8) {
    bfly8<DIR>(v);
  } else if constexpr (K == 3) {
    bfly3<DIR>(v);
  } else {
    // K = K1*K2 (16 = 4*4, 32 = 8*4, 12 = 4*3, 24 = 8*3): element K2*a + b ; output c + K1*d
    constexpr int K1 = dft_split<K>();
    constexpr int K2 = K / K1;
    C Y[K2][K1];
#pragma unroll
    for (int b = 0; b < K2; ++b) {
      C t[K1];
#pragma unroll
      for (int a = 0; a < K1; ++a) t[a] = v[K2 * a + b];
      dftr<K1, DIR>(t);
#pragma unroll
      for (int c = 0; c < K1; ++c) Y[b][c] = cmul_wk<K, DIR>(t[c], b * c);
    }
#pragma unroll
    for (int c = 0; c < K1; ++c) {
      C t[K2];
#pragma unroll
      for (int b = 0; b < K2; ++b) t[b] = Y[b][c];
      dftr<K2, DIR>(t);
#pragma unroll
      for (int d = 0; d < K2; ++d) v[c + K1 * d] = t[d];
    }
  }
}

// DFT of K points whose upper half v[K/2..K-1] is zero (not read): the
// zero-padded half of a forward DDA transform.  Same output as dftr<K>.
template <int K, int DIR, typename C> __device__ __forceinline__ void dftr_h(C* v) {
  if constexpr (K == 2) {
    v[1] = v[0];
  } else if constexpr (K == 4) {
    const C a = v[0], b = v[1];
    v[0] = vadd(a, b);
    v[2] = vsub(a, b);
    v[1] = addrot<DIR>(a, b);  // a + DIR*i*b
    v[3] = subrot<DIR>(a, b);
  } else if constexpr (K == 8) {
    C e[4] = {v[0], v[2], v[0], v[0]};
    C o[4] = {v[1], v[3], v[1], v[1]};
    dftr_h<4, DIR>(e);
    dftr_h<4, DIR>(o);
    const C t1 = w8_1<DIR>(o[1]), t3 = w8_3<DIR>(o[3]);
    v[0] = vadd(e[0], o[0]);
    v[4] = vsub(e[0], o[0]);
    v[1] = vadd(e[1], t1);
    v[5] = vsub(e[1], t1);
    v[2] = addrot<DIR>(e[2], o[2]);
    v[6] = subrot<DIR>(e[2], o[2]);
    v[3] = vadd(e[3], t3);
    v[7] = vsub(e[3], t3);
  } else {
    // K = K1*K2, element K2*a + b is zero for a >= K1/2
    constexpr int K1 = dft_split<K>();
    constexpr int K2 = K / K1;
    C Y[K2][K1];
#pragma unroll
    for (int b = 0; b < K2; ++b) {
      C t[K1];
#pragma unroll
      for (int a = 0; a < K1 / 2; ++a) t[a] = v[K2 * a + b];
      dftr_h<K1, DIR>(t);
#pragma unroll
      for (int c = 0; c < K1; ++c) Y[b][c] = cmul_wk<K, DIR>(t[c], b * c);
    }
#pragma unroll
    for (int c = 0; c < K1; ++c) {
      C t[K2];
#pragma unroll
      for (int b = 0; b < K2; ++b) t[b] = Y[b][c];
      dftr<K2, DIR>(t);
#pragma unroll
      for (int d = 0; d < K2; ++d) v[c + K1 * d] = t[d];
    }
  }
}

// Transpose scratch of one line: T rows of E elements.  Row stride E + 1, or
// E + 2 with PAIR (even, so that element pairs are 16-byte aligned and each
// pair is written with one 128-bit store).
template <int E, bool PAIR = false> constexpr int row_stride() { return PAIR ? E + 2 : E + 1; }
template <int E, int T, bool PAIR = false> constexpr int line_scratch() { return T * row_stride<E, PAIR>() + 2; }

// Line stride (complex elements) for L lines per block whose threads are
// interleaved line-fastest (column passes) or thread-fastest (row passes): the
// smallest stride >= T*rowstride for which the transpose is free of
// shared-memory bank conflicts where one exists.  Reads: the 16 lanes of a
// half-warp load 8-byte elements at s*rs + t and must hit 16 distinct 8-byte
// bank pairs.  Writes: without pair, the 16 lanes of a half-warp store 8 bytes
// at t*rs + p; with pair (even strides only), the 8 lanes of a quarter-warp
// store 16 bytes and must hit 8 distinct 16-byte bank groups.
inline int line_stride(int E, int T, int L, bool line_fastest, bool pair = false) {
  const int RS = pair ? E + 2 : E + 1;
  const int base = T * RS;
  auto lane_lt = [&](int lane, int& l, int& t) {
    if (line_fastest) { l = lane % L; t = lane / L; } else { t = lane % T; l = lane / T; }
    return l < L && t < T;
  };
  for (int pad = 0; pad < 64; pad += pair ? 2 : 1) {
    const int LS = base + pad;
    bool ok = true;
    const int wl = pair ? 8 : 16;  // lanes per write wavefront
    for (int q = 0; q < 32 / wl && ok; ++q) {
      unsigned used = 0;
      for (int k = 0; k < wl && ok; ++k) {
        int l, t;
        if (!lane_lt(wl * q + k, l, t)) continue;
        const int a = l * LS + t * RS;
        const int g = pair ? (a / 2) & 7 : a & 15;
        if (used & (1u << g)) ok = false;
        used |= 1u << g;
      }
    }
    for (int h = 0; h < 2 && ok; ++h) {
      unsigned used = 0;
      for (int k = 0; k < 16 && ok; ++k) {
        int l, t;
        if (!lane_lt(16 * h + k, l, t)) continue;
        const int a = (l * LS + t) & 15;
        if (used & (1u << a)) ok = false;
        used |= 1u << a;
      }
    }
    if (ok) return LS;
  }
  return base + (pair ? 2 : 1);
}

// Four-step twiddles W^(t p), p = 1..E-1, of thread t for DIR: the powers of
// two come from the table tw[m] = exp(-2*pi*i*m/N), the others are products
// of at most four of them (fewer shared-memory loads).  w[0] is not set.
template <int E, int DIR, typename C>
__device__ __forceinline__ void line_twiddles(C (&w)[E], int t, const C* __restrict__ tw) {
#pragma unroll
  for (int b = 1; b < E; b <<= 1) w[b] = twid<DIR>(tw, t * b);
#pragma unroll
  for (int p = 3; p < E; ++p) {
    const int hb = 1 << (31 - __clz(p));  // highest set bit of p
    if (p != hb) w[p] = cmul(w[hb], w[p - hb]);
  }
}

// a * conj(w)
template <typename C> __device__ __forceinline__ C cmulc(C a, C w) {
  return mk2<C>(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}

// One length-E*T transform of the line held in v by thread t (0 <= t < T),
// with the thread's twiddles w from line_twiddles: those of DIR, or with
// CONJW those of -DIR, applied conjugated (so one set serves a forward and an
// inverse transform; both give the same products as a set built for DIR).
// `sl` is this line's shared scratch.  BLOCK_SYNC selects __syncthreads (line
// spread over warps) or __syncwarp.  HALF_IN: elements t + T*i with i >= E/2
// (the upper half of the line) are zero and are not read.  PAIR: transpose
// rows of stride E + 2 written with 128-bit stores (complex-float lines; the
// line stride must come from line_stride(..., pair = true)).
template <int E, int T, int DIR, bool BLOCK_SYNC, bool HALF_IN = false, bool PAIR = false, bool CONJW = false,
          typename C>
__device__ __forceinline__ void line_fft_w(C (&v)[E], C* sl, int t, const C (&w)[E]) {
  constexpr int M = E / T;
  static_assert(M * T == E && M >= 1, "E must be a multiple of T");
  if constexpr (HALF_IN) dftr_h<E, DIR>(v); else dftr<E, DIR>(v);
#pragma unroll
  for (int p = 1; p < E; ++p) v[p] = CONJW ? cmulc(v[p], w[p]) : cmul(v[p], w[p]);
  constexpr bool P2 = PAIR && sizeof(C) == 8;
  constexpr int RS = row_stride<E, P2>();
  if constexpr (P2) {
#pragma unroll
    for (int p = 0; p < E; p += 2)
      *reinterpret_cast<float4*>(sl + t * RS + p) = make_float4(v[p].x, v[p].y, v[p + 1].x, v[p + 1].y);
  } else {
#pragma unroll
    for (int p = 0; p < E; ++p) sl[t * RS + p] = v[p];
  }
  if (BLOCK_SYNC) __syncthreads(); else __syncwarp();
#pragma unroll
  for (int j = 0; j < M; ++j) {
    C u[T];
#pragma unroll
    for (int s = 0; s < T; ++s) u[s] = sl[s * RS + t + T * j];
    dftr<T, DIR>(u);
#pragma unroll
    for (int q = 0; q < T; ++q) v[j + M * q] = u[q];
  }
  if (BLOCK_SYNC) __syncthreads(); else __syncwarp();
}

// One length-E*T transform with its own twiddles (`tw` as in line_twiddles).
template <int E, int T, int DIR, bool BLOCK_SYNC, bool HALF_IN = false, bool PAIR = false, typename C>
__device__ __forceinline__ void line_fft(C (&v)[E], C* sl, int t, const C* __restrict__ tw) {
  C w[E];
  line_twiddles<E, DIR>(w, t, tw);
  line_fft_w<E, T, DIR, BLOCK_SYNC, HALF_IN, PAIR>(v, sl, t, w);
}

// (E, T) shape for a supported power-of-two length, E*T = N
template <int N> struct RegShape;
template <> struct RegShape<16> { static constexpr int E = 4, T = 4; };
template <> struct RegShape<32> { static constexpr int E = 8, T = 4; };
template <> struct RegShape<64> { static constexpr int E = 8, T = 8; };
template <> struct RegShape<128> { static constexpr int E = 16, T = 8; };
template <> struct RegShape<256> { static constexpr int E = 16, T = 16; };
template <> struct RegShape<512> { static constexpr int E = 32, T = 16; };
// 3 * 2^k lengths (x-first pipeline only)
template <> struct RegShape<48> { static constexpr int E = 12, T = 4; };
template <> struct RegShape<96> { static constexpr int E = 24, T = 4; };
template <> struct RegShape<192> { static constexpr int E = 24, T = 8; };

inline bool reg_supported(int n) { return n == 16 || n == 32 || n == 64 || n == 128 || n == 256 || n == 512; }
inline bool xreg_supported(int n) { return reg_supported(n) || n == 48 || n == 96 || n == 192; }
// threads per line of the register shape of length n (RegShape<n>::T)
inline int reg_threads(int n) {
  switch (n) {
    case 16: case 32: case 48: case 96: return 4;
    case 64: case 128: case 192: return 8;
    default: return 16;
  }
}

}  // namespace ddb
