// x-first, transposed-layout MATVEC pipeline for power-of-two grids (sm_100a).
//
// Same operator as matvec.cu (cprod_cuda.f90:446-607 / ddscat_matvec_cuda.cu:
// 104-118), organised so that every pass transforms along the contiguous axis
// of its input with the T threads of a line inside one warp (register line
// FFTs, fftreg.cuh), and the axis change is done by a shared-memory tile
// transpose on the load or store side, keeping global accesses in 128-byte
// segments (at the 256- and 512-point shapes the tiles move between shared and
// global memory by the tensor memory accelerator):
//   XF : x (compact or full) rows  -> x-FFT(+i), pad-skip -> A[c][iz][kx][iy]
//   YF : A y-rows (n_y)            -> y-FFT(+i)           -> B[c][kx][ky][iz]
//   ZG : B z-rows (n_z)            -> z-FFT(+i) * Green * z-FFT(-i), keep n_z
//   YI : B (transposed load)       -> y-FFT(-i), keep n_y -> A
//   XI : A (transposed load)       -> x-FFT(-i), keep n_x -> finish -> y
// Optionally (DDSCAT_B200_FUSEXY=1; FP32, M_x and M_y up to 256, FFT3D build)
// the x and y passes of a z plane run fused in one cluster of four CTAs (XYF,
// XYI below): the plane meets in distributed shared memory instead of an HBM
// round trip of A, and B is laid out [c][kx][iz][ky] for them.
// The Green octant is stored z-fastest, [irx][iry][irz][6], so a z-line reads
// contiguous 48-byte records.  kx_zg3 (the ZG pass for E <= 16, FP32) keeps
// the three components of a z position in one thread and reads its records
// straight from global memory, its grid RHS-fastest so that consecutive blocks
// reuse the octant lines from L2; kx_zg3r (the default for batches of 4 RHS
// or more, IPBC = 0) stages a block's octant lines in shared memory once and
// runs the z pass for a chunk of RHS with them; kx_zg (larger E, FP64) loads
// each record once for kz and its mirror M_z - kz and exchanges the
// components through shared memory.  Twiddles are read from global memory
// (L1/L2 resident tables).  The middle passes run over kx batches (all of M_x
// for the FFT3D build, a few columns for the SLICES build).
#include <algorithm>
#include <cstdlib>
#include <cooperative_groups.h>
#include <cuda.h>
#include <cudaTypedefs.h>
#include "engine.h"
#include "fftreg.cuh"

namespace ddb {

template <typename T> struct XParams {
  // B as a 2-D tensor of rows of n_z 8-byte complex floats, box {16, 256},
  // 128-byte swizzle: the tiles of the 256-point y passes (tma != 0)
  alignas(64) CUtensorMap tmB;
  // A as rows of n_y complex floats, box {16, 256}: the tiles of the 256-point
  // x passes (tma_x != 0)
  alignas(64) CUtensorMap tmA;
  int tma;
  int tma_x;
  int* err;  // status word (Engine::d_err)
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
  const int* rowq;  // compact index of the first occupied site of each x row
  const int* mask;
  int rhs0;
  cplx<T>* A;  // [rl][c][iz][kx][iy]
  size_t A_rs;
  cplx<T>* B;  // [rb][c][kxl][ky][iz] for kx in [kx0, kx0 + nkx); fused xy passes: [rb][c][kx][iz][ky]
  int kx0, nkx, b_rhs0;
  int nrb_mid;  // RHS of the current middle-stage batch
  int zg_rch;   // RHS per ZG3R block (blockIdx.y = chunk)
  const cplx<T>* green;  // [irx][iry][irz][6] (IPBC=0) or [kx][ky][kz][6] (IPBC=1)
  int ipbc;
  const cplx<T>* twx;
  const cplx<T>* twy;
  const cplx<T>* twz;
  int lsx, lsy, lsz;  // line strides of the x, y, z passes
  int tlx;            // tile / line scratch elements of the x passes
  T inv_ngrid;
  double2* dot_out;  // optional fused sum of x*y per RHS (MvArgs::dot_out)
  double2* dot_part;
  unsigned* dot_cnt;
  int dot_k;
};

template <typename T> __device__ __forceinline__ bool xoff(const XParams<T>& P, int rl) {
  return P.mask != nullptr && P.mask[P.rhs0 + rl] == 0;
}


// Compile-time shape of a pass over the padded axis length N >= 2n: E elements
// per thread, TT threads per line, H = E/2 elements per thread in the first
// half N/2 >= n (those with index >= n are masked), RL lines per 256-thread
// row block.
template <int N> struct XShape {
  static constexpr int E = RegShape<N>::E, TT = RegShape<N>::T, H = E / 2;
  static constexpr int RL = 256 / TT;
  static constexpr int RZ = (128 / TT) > 1 ? 128 / TT : 1;  // ZG lines per block (3*TT*RZ threads)
  static constexpr int ZG_MINB = E >= 32 ? 1 : (E >= 24 ? 2 : 3);  // ZG blocks per SM the registers must allow (FP32)
  static constexpr bool PAIR = TT >= 8;                      // 128-bit transpose stores (conflict-free for TT >= 8)
};

// ---- tensor-memory-accelerator tiles of the 256-point y passes (FP32)
// A y-pass tile holds 256 rows (ky) of 16 consecutive z positions: 128 bytes
// per row, stored with the 128-byte swizzle (16-byte chunk j of row r at chunk
// j ^ (r & 7)), the layout a box of {16, 256} 8-byte elements has in shared
// memory.  The tile base is 1024-byte aligned.  Threads write and read it
// through tma_slot; the tensor map covers this GPU's own B buffer and no
// multicast is used.
constexpr int TMA_ROWS = 256, TMA_COLS = 16;
constexpr unsigned TMA_TILE_BYTES = TMA_ROWS * TMA_COLS * 8;
constexpr int TMA_WAIT_POLLS = 1 << 24;  // bounded wait for a tile load (seconds at most)
__device__ __forceinline__ int tma_slot(int r, int col) {
  return r * TMA_COLS + (((col >> 1) ^ (r & 7)) << 1) + (col & 1);
}
__device__ __forceinline__ float2* tma_tile(unsigned char* smem) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(smem);
  return reinterpret_cast<float2*>((a + 1023) & ~(uintptr_t)1023);
}
// A tile of N = 256 or 512 rows is N/256 boxes of 256 rows, each 32 KB and
// 1024-byte aligned (the swizzle phase r & 7 is the same in every box).
template <int N> constexpr bool tma_rows_ok() { return N == 256 || N == 512; }
// store the tile's boxes at (x = inner position, y = first row) of the map;
// the issuing thread waits until the copies have read the tile (the CTA keeps
// its shared memory)
template <int N> __device__ __forceinline__ void tma_store_tile(const CUtensorMap* map, const float2* tile, int x, int y) {
#pragma unroll
  for (int b = 0; b < N / TMA_ROWS; ++b)
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(map), "r"(x),
                 "r"(y + b * TMA_ROWS), "r"(smem_addr(tile + (size_t)b * TMA_ROWS * TMA_COLS))
                 : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// load the tile's boxes, completing on bar (which expects N/256 * 32 KB)
template <int N>
__device__ __forceinline__ void tma_load_tile(const CUtensorMap* map, float2* tile, int x, int y, uint64_t* bar) {
#pragma unroll
  for (int b = 0; b < N / TMA_ROWS; ++b)
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(tile + (size_t)b * TMA_ROWS * TMA_COLS)),
        "l"(map), "r"(x), "r"(y + b * TMA_ROWS), "r"(smem_addr(bar))
        : "memory");
}

// Tile <-> global moves of the row passes: N rows of RL consecutive elements
// (row stride ld in global, RL+1 in the tile), two elements per 16-byte access.
// Rows hold `valid` elements (RL or fewer at the grid edge; always even,
// since every axis length n is even here and RL is even).  The global base and
// ld are even in elements, so every pair is 16-byte aligned.
template <int RL, int N, typename C>
__device__ __forceinline__ void store_pairs(C* g, int ld, int valid, const C* tile) {
  constexpr int RP = RL / 2;
#pragma unroll 4
  for (int u = threadIdx.x; u < N * RP; u += 256) {
    const int r = u / RP, ll = 2 * (u % RP);
    if (ll < valid) {
      const C a = tile[r * (RL + 1) + ll], b = tile[r * (RL + 1) + ll + 1];
      if constexpr (sizeof(C) == 8) {
        *reinterpret_cast<float4*>(g + (size_t)r * ld + ll) = make_float4(a.x, a.y, b.x, b.y);
      } else {
        g[(size_t)r * ld + ll] = a;
        g[(size_t)r * ld + ll + 1] = b;
      }
    }
  }
}
// Global -> tile move of the column passes (the inverse of store_pairs),
// staged through registers: all of a thread's 16-byte loads are issued before
// its shared-memory stores (one memory round trip per block, fewer
// instructions than 8-byte cp.async copies).  Rows hold `valid` elements, an
// even count, and the global base and ld are even in elements, so every
// complex-float pair is 16-byte aligned.
template <int RL, int N, typename C>
__device__ __forceinline__ void load_tile_pairs(const C* g, int ld, int valid, C* tile) {
  static_assert((N * RL / 2) % 256 == 0, "tiles of whole 256-thread rounds");
  if constexpr (sizeof(C) == 8) {
    constexpr int RP = RL / 2, K = N * RP / 256;
    float4 q[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int u = threadIdx.x + 256 * k, r = u / RP, ll = 2 * (u - r * RP);
      q[k] = ll < valid ? __ldg(reinterpret_cast<const float4*>(g + (size_t)r * ld + ll))
                        : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int u = threadIdx.x + 256 * k, r = u / RP, ll = 2 * (u - r * RP);
      tile[r * (RL + 1) + ll] = mk<C>(q[k].x, q[k].y);
      tile[r * (RL + 1) + ll + 1] = mk<C>(q[k].z, q[k].w);
    }
  } else {  // complex double: one 16-byte element per load
    constexpr int K = N * RL / 256;
    C q[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int u = threadIdx.x + 256 * k, r = u / RL, ll = u - r * RL;
      q[k] = ll < valid ? g[(size_t)r * ld + ll] : mk<C>(0, 0);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int u = threadIdx.x + 256 * k, r = u / RL, ll = u - r * RL;
      tile[r * (RL + 1) + ll] = q[k];
    }
  }
}

// Asynchronous copy of cnt (<= MAXC) contiguous elements from global to shared
// memory with the whole 256-thread block (completed by cp_async_wait_all).
template <int MAXC, typename C> __device__ __forceinline__ void stage_chunk_async(C* dst, const C* src, int cnt) {
#pragma unroll
  for (int k = 0; k < (MAXC + 255) / 256; ++k) {
    const int u = threadIdx.x + 256 * k;
    if (u < cnt) {
      if constexpr (sizeof(C) == 8) cp_async8(dst + u, src + u, true);
      else cp_async16(dst + u, src + u);
    }
  }
}

// ------------------------------------------------------------- XF: x forward
// block: RL rows (iy) x TT threads, thread-fastest; grid (ceil(ny/RL), nz, 3*nr)
template <typename T, int N> __global__ void __launch_bounds__(256) kx_xf(const __grid_constant__ XParams<T> P) {
  using C = cplx<T>;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RL = S_::RL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* tile = reinterpret_cast<C*>(smem_raw);   // [kx][RL+1], aliases the line scratch
  C* lines = reinterpret_cast<C*>(smem_raw);  // RL * lsx
  const int iy0 = blockIdx.x * RL, iy = iy0 + l, iz = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3);
  if (xoff(P, rl)) return;
  const int S = P.io_full ? P.nat : P.nat0;
  const C* x = P.x + (size_t)rl * P.x_rs + (size_t)c * S;
  const int jrow = P.nx * (iy + P.ny * iz);
  C v[E];
  if (P.io_full) {
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = iy < P.ny && t + TT * i < P.nx ? x[jrow + t + TT * i] : mk<C>(0, 0);  // ix < nx <= N/2
  } else {
    // the block's rows hold one contiguous compact range [q0, q0 + cnt): copy
    // it to shared memory (coalesced) while the inv lookups are in flight,
    // then gather from there
    const int r0 = iy0 + P.ny * iz, nrows = min(RL, P.ny - iy0);
    const int q0 = P.rowq[r0], cnt = P.rowq[r0 + nrows] - q0;
    int qi[H];
#pragma unroll
    for (int i = 0; i < H; ++i) qi[i] = iy < P.ny && t + TT * i < P.nx ? P.inv[jrow + t + TT * i] : -1;
    C* chunk = lines;  // at most RL*nx elements; consumed before the FFT uses the scratch
    stage_chunk_async<RL * (N / 2)>(chunk, x + q0, cnt);
    cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = qi[i] >= 0 ? chunk[qi[i] - q0] : mk<C>(0, 0);
    __syncthreads();
  }
  if (P.conj) {
#pragma unroll
    for (int i = 0; i < H; ++i) v[i].y = -v[i].y;
  }
  line_fft<E, TT, +1, false, true, S_::PAIR>(v, lines + (size_t)l * P.lsx, t, P.twx);
  __syncthreads();  // all line scratch consumed before the tile reuses it
  if constexpr (tma_rows_ok<N>() && RL == TMA_COLS && sizeof(C) == 8) {
    if (P.tma_x) {
      // swizzled tile, then one tensor store of its 256 x 16 elements (rows
      // beyond n_y are clipped by the map)
      C* tt = tma_tile(smem_raw);
#pragma unroll
      for (int i = 0; i < E; ++i) tt[tma_slot(t + TT * i, l)] = v[i];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0) tma_store_tile<N>(&P.tmA, tt, iy0, ((rl * 3 + c) * P.nz + iz) * P.Mx);
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < E; ++i) tile[(t + TT * i) * (RL + 1) + l] = v[i];
  __syncthreads();
  C* A = P.A + (size_t)rl * P.A_rs + ((size_t)(c * P.nz + iz) * P.Mx) * P.ny + iy0;
  store_pairs<RL, N>(A, P.ny, P.ny - iy0, tile);
}

// ------------------------------------------------------------- YF: y forward
// block: RL z-lines (iz) x TT; grid (ceil(nz/RL), nkx, 3*nrb)
template <typename T, int N> __global__ void __launch_bounds__(256) kx_yf(const __grid_constant__ XParams<T> P) {
  using C = cplx<T>;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RL = S_::RL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* tile = reinterpret_cast<C*>(smem_raw);
  C* lines = reinterpret_cast<C*>(smem_raw);
  const int iz0 = blockIdx.x * RL, iz = iz0 + l, kxl = blockIdx.y, kx = P.kx0 + kxl;
  const int rb = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3), rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;
  const C* A = P.A + (size_t)rl * P.A_rs + ((size_t)(c * P.nz + iz) * P.Mx + kx) * P.ny;
  C v[E];
  const bool zin = iz < P.nz;
#pragma unroll
  for (int i = 0; i < H; ++i) v[i] = zin && t + TT * i < P.ny ? A[t + TT * i] : mk<C>(0, 0);  // iy < ny <= N/2
  line_fft<E, TT, +1, false, true, S_::PAIR>(v, lines + (size_t)l * P.lsy, t, P.twy);
  __syncthreads();
  if constexpr (tma_rows_ok<N>() && RL == TMA_COLS && sizeof(C) == 8) {
    if (P.tma) {
      // swizzled tile, then one tensor store of its 256 x 16 elements (z
      // positions beyond n_z are clipped by the map)
      C* tt = tma_tile(smem_raw);
#pragma unroll
      for (int i = 0; i < E; ++i) tt[tma_slot(t + TT * i, l)] = v[i];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (threadIdx.x == 0) tma_store_tile<N>(&P.tmB, tt, iz0, ((rb * 3 + c) * P.nkx + kxl) * P.My);
      return;
    }
  }
#pragma unroll
  for (int i = 0; i < E; ++i) tile[(t + TT * i) * (RL + 1) + l] = v[i];
  __syncthreads();
  C* B = P.B + ((size_t)(rb * 3 + c) * P.nkx + kxl) * (size_t)P.My * P.nz + iz0;
  store_pairs<RL, N>(B, P.nz, P.nz - iz0, tile);
}

// Green record at (kx, ky, kz) for the z-fastest layout, without the kz sign.
template <typename T>
__device__ __forceinline__ const cplx<T>* green_rec(const XParams<T>& P, int kx, int ky, int kz, T& sxy, T& sxz,
                                                    T& syz) {
  size_t b;
  if (P.ipbc == 0) {
    const T sx = 2 * kx <= P.Mx ? (T)1 : (T)-1, sy = 2 * ky <= P.My ? (T)1 : (T)-1;
    const int irx = min(kx, P.Mx - kx), iry = min(ky, P.My - ky);
    b = ((size_t)irx * (P.My / 2 + 1) + iry) * (P.Mz / 2 + 1) + kz;
    sxy = sx * sy; sxz = sx; syz = sy;  // times sz, applied by the caller
  } else {
    b = ((size_t)kx * P.My + ky) * P.Mz + kz;
    sxy = sxz = syz = (T)1;
  }
  return P.green + 6 * b;
}

template <typename T> __device__ __forceinline__ void load_rec(const cplx<T>* gp, cplx<T> a[6]) {
  if constexpr (sizeof(cplx<T>) == 8) {
    const float4* g4 = reinterpret_cast<const float4*>(gp);
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
}

template <typename C, typename R>
__device__ __forceinline__ void green_apply(const C a[6], R sxy, R sxz, R syz, C& px, C& py, C& pz) {
  const C a12 = cscale(a[1], sxy), a13 = cscale(a[2], sxz), a23 = cscale(a[4], syz);
  const C x = px, y = py, z = pz;
  px = cadd(cadd(cmul(a[0], x), cmul(a12, y)), cmul(a13, z));
  py = cadd(cadd(cmul(a12, x), cmul(a[3], y)), cmul(a23, z));
  pz = cadd(cadd(cmul(a13, x), cmul(a23, y)), cmul(a[5], z));
}

// y = G x for one octant record a = (xx, xy, xz, yy, yz, zz) with the
// off-diagonal signs SXY, SXZ, SYZ (+1 or -1, compile-time, so they fold into
// the operands): each real and imaginary output is one multiply and five
// fused multiply-adds.
template <int SXY, int SXZ, int SYZ, typename C>
__device__ __forceinline__ void green_apply_s(const C a[6], C& px, C& py, C& pz) {
  using R = decltype(px.x);
  const C x = px, y = py, z = pz;
  const R kxy = (R)SXY, kxz = (R)SXZ, kyz = (R)SYZ;
  // row x: a0 x + SXY a1 y + SXZ a2 z
  px.x = fma(kxz * a[2].x, z.x, fma(-kxz * a[2].y, z.y, fma(kxy * a[1].x, y.x, fma(-kxy * a[1].y, y.y,
         fma(a[0].x, x.x, -a[0].y * x.y)))));
  px.y = fma(kxz * a[2].x, z.y, fma(kxz * a[2].y, z.x, fma(kxy * a[1].x, y.y, fma(kxy * a[1].y, y.x,
         fma(a[0].x, x.y, a[0].y * x.x)))));
  // row y: SXY a1 x + a3 y + SYZ a4 z
  py.x = fma(kyz * a[4].x, z.x, fma(-kyz * a[4].y, z.y, fma(a[3].x, y.x, fma(-a[3].y, y.y,
         fma(kxy * a[1].x, x.x, -kxy * a[1].y * x.y)))));
  py.y = fma(kyz * a[4].x, z.y, fma(kyz * a[4].y, z.x, fma(a[3].x, y.y, fma(a[3].y, y.x,
         fma(kxy * a[1].x, x.y, kxy * a[1].y * x.x)))));
  // row z: SXZ a2 x + SYZ a4 y + a5 z
  pz.x = fma(a[5].x, z.x, fma(-a[5].y, z.y, fma(kyz * a[4].x, y.x, fma(-kyz * a[4].y, y.y,
         fma(kxz * a[2].x, x.x, -kxz * a[2].y * x.y)))));
  pz.y = fma(a[5].x, z.y, fma(a[5].y, z.x, fma(kyz * a[4].x, y.y, fma(kyz * a[4].y, y.x,
         fma(kxz * a[2].x, x.y, kxz * a[2].y * x.x)))));
}

// Offset of z position 0 of line p = kxl*My + ky in one component of B, and
// the z stride: [kxl][ky][iz] (five-pass schedule, BTY = 0) or [kx][iz][ky]
// (the fused xy passes, BTY = M_y: a compile-time stride keeps the z offsets
// immediate).
template <int BTY, typename T> __device__ __forceinline__ size_t zline_base(const XParams<T>& P, int p) {
  if constexpr (BTY > 0) {
    const int kxl = p / BTY;
    return (size_t)kxl * P.nz * BTY + (p - kxl * BTY);
  } else {
    return (size_t)p * P.nz;
  }
}
template <int BTY> constexpr int zline_stride() { return BTY > 0 ? BTY : 1; }

// ------------------------------------------------------------- ZG: z * Green * z^-1
// block: RZ lines x TT threads x 3 components, thread-fastest within a line;
// lines are (kx, ky) pairs p = kxl*My + ky.  grid (nrb, ceil(nkx*My/RZ))
template <typename T, int N, int BTY = 0>
__global__ void __launch_bounds__(3 * XShape<N>::TT * XShape<N>::RZ, sizeof(T) == 8 ? 1 : XShape<N>::ZG_MINB)
    kx_zg(XParams<T> P) {
  using C = cplx<T>;
  using R = T;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RL = S_::RZ;
  constexpr int GT = 3 * TT;  // Green-phase threads per line
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = (threadIdx.x / TT) % RL, c = threadIdx.x / (TT * RL);
  C* lines = reinterpret_cast<C*>(smem_raw);  // [3][RL][lsz]
  C* my = lines + (size_t)(c * RL + l) * P.lsz;
  const int rb = blockIdx.x, rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;
  const int nlines = P.nkx * P.My;
  const int p = blockIdx.y * RL + l;
  const bool live = p < nlines;
  constexpr int zs = zline_stride<BTY>();
  C* row = P.B + ((size_t)(rb * 3 + c) * P.nkx) * (size_t)P.My * P.nz + zline_base<BTY>(P, live ? p : 0);
  C v[E];
#pragma unroll
  for (int i = 0; i < H; ++i)
    v[i] = live && t + TT * i < P.nz ? row[(t + TT * i) * zs] : mk<C>(0, 0);  // iz < nz <= N/2
  line_fft<E, TT, +1, false, true, S_::PAIR>(v, my, t, P.twz);
#pragma unroll
  for (int i = 0; i < E; ++i) my[t + TT * i] = v[i];
  __syncthreads();
  // Green: GT threads per line, kz = 0..N/2; the record serves kz and N - kz
  {
    const int gl = threadIdx.x / GT, gk = threadIdx.x - GT * (threadIdx.x / GT);
    const int pl = blockIdx.y * RL + gl;
    if (pl < nlines) {
      const int kxl = pl / P.My;  // My need not be a power of two (3 * 2^k lengths)
      const int kx = P.kx0 + kxl, ky = pl - kxl * P.My;
      C* L0 = lines + (size_t)gl * P.lsz;
      C* L1 = L0 + (size_t)RL * P.lsz;
      C* L2 = L1 + (size_t)RL * P.lsz;
      if (P.ipbc == 0) {
        R sxy, sxz, syz;
        const C* rec0 = green_rec(P, kx, ky, 0, sxy, sxz, syz);
        // records kz = gk + GT*j: up to 3 loads in flight before the first use
        constexpr int NIT = (N / 2 + GT) / GT;
#pragma unroll
        for (int j0 = 0; j0 < NIT; j0 += 3) {
          C a[3][6];
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int kz = gk + GT * (j0 + j);
            if (j0 + j < NIT && kz <= N / 2) load_rec<T>(rec0 + 6 * kz, a[j]);
          }
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const int kz = gk + GT * (j0 + j);
            if (j0 + j < NIT && kz <= N / 2) {
              green_apply(a[j], sxy, sxz, syz, L0[kz], L1[kz], L2[kz]);  // kz <= nz: sz = +1
              const int km = N - kz;
              if (kz > 0 && km != kz) green_apply(a[j], sxy, -sxz, -syz, L0[km], L1[km], L2[km]);  // sz = -1
            }
          }
        }
      } else {
        for (int kz = gk; kz < N; kz += GT) {
          R sxy, sxz, syz;
          C a[6];
          load_rec<T>(green_rec(P, kx, ky, kz, sxy, sxz, syz), a);
          green_apply(a, sxy, sxz, syz, L0[kz], L1[kz], L2[kz]);
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < E; ++i) v[i] = my[t + TT * i];
  __syncwarp();
  line_fft<E, TT, -1, false, false, S_::PAIR>(v, my, t, P.twz);
  if (live) {
#pragma unroll
    for (int i = 0; i < H; ++i)
      if (t + TT * i < P.nz) row[(t + TT * i) * zs] = v[i];  // keep iz < nz
  }
}

// ------------------------------------------------------------- ZG3: z * Green * z^-1, components in registers
// Each thread holds the same z positions of all three components of its
// (kx, ky) line, so the Green multiply runs in registers: shared memory only
// carries the FFT transposes (half the shared-memory traffic of kx_zg, no
// block barriers).  The Green octant records (48 bytes, kz > N/2 reads the
// record of N - kz with the kz sign) come straight from global memory, four
// per thread at a time; consecutive blocks work on the same lines for
// successive RHS (the grid runs RHS-fastest), so the records are L2 hits.
// Staging the block's octant lines in shared memory by bulk asynchronous
// copies instead measured 7 % slower at 128^3 (66 KB more shared memory per
// block, a smaller L1).  For E <= 16 (registers: 3E complex per thread).
// block: RZ lines x TT threads, thread-fastest; grid (nrb, ceil(nkx*My/RZ))
// shared memory: FFT scratch [RZ][lsz]
template <int N> struct Z3Shape {
  static constexpr int RZ = 128 / XShape<N>::TT;  // lines per 128-thread block
  static constexpr bool OK = XShape<N>::E <= 16;
};

// The Green multiply of kx_zg3 on data whose x and y components carry the
// line signs sx (kx) and sy (ky) already (the off-diagonal signs of the octant,
// cu:112, are s_a s_b, i.e. G = D G' D with D = diag(sx, sy, sz)); what is left
// is the kz sign of the xz and yz entries, compile-time for every element but
// the one at i = E/2, whose kz = N/2 + t has sign +1 only for t = 0.
template <int N, int TT, int E, typename C>
__device__ __forceinline__ void zg3_green(const C* rec0, int t, C (&v)[3][E]) {
  constexpr int GB = 4;  // records in flight per thread (2 measured 9 % slower at 128^3)
#pragma unroll
  for (int i0 = 0; i0 < E; i0 += GB) {
    C a[GB][6];
#pragma unroll
    for (int j = 0; j < GB; ++j) {
      const int kz = t + TT * (i0 + j);
      load_rec<decltype(a[0][0].x)>(rec0 + 6 * (kz <= N / 2 ? kz : N - kz), a[j]);
    }
#pragma unroll
    for (int j = 0; j < GB; ++j) {
      const int i = i0 + j;
      // i is a constant after unrolling: these tests fold
      if (TT * i + TT - 1 <= N / 2) {
        green_apply_s<1, 1, 1>(a[j], v[0][i], v[1][i], v[2][i]);
      } else if (TT * i > N / 2) {
        green_apply_s<1, -1, -1>(a[j], v[0][i], v[1][i], v[2][i]);
      } else {
        if (t + TT * i <= N / 2) green_apply_s<1, 1, 1>(a[j], v[0][i], v[1][i], v[2][i]);
        else green_apply_s<1, -1, -1>(a[j], v[0][i], v[1][i], v[2][i]);
      }
    }
  }
}

template <typename T, int N, int BTY = 0> __global__ void __launch_bounds__(128, 3) kx_zg3(XParams<T> P) {
  using C = cplx<T>;
  using R = T;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H;
  static_assert(Z3Shape<N>::OK, "kx_zg3 holds 3*E complex values per thread");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* my = reinterpret_cast<C*>(smem_raw) + (size_t)l * P.lsz;
  const int rb = blockIdx.x, rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;
  const int nlines = P.nkx * P.My;
  const int p = blockIdx.y * Z3Shape<N>::RZ + l;
  const bool live = p < nlines;
  const size_t cs = (size_t)nlines * P.nz;  // component stride of B
  constexpr int zs = zline_stride<BTY>();
  C* row = P.B + (size_t)rb * 3 * cs + zline_base<BTY>(P, live ? p : 0);
  const int kxl = p / P.My;
  const int kx = P.kx0 + kxl, ky = p - kxl * P.My;
  // the octant's line signs sx (kx) and sy (ky) of cu:112, applied to the x and
  // y components on the way in and out (the z transforms are linear)
  const R sx = P.ipbc == 0 && 2 * kx > P.Mx ? (R)-1 : (R)1, sy = P.ipbc == 0 && 2 * ky > P.My ? (R)-1 : (R)1;
  C v[3][E];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R sc = c == 0 ? sx : (c == 1 ? sy : (R)1);
#pragma unroll
    for (int i = 0; i < H; ++i)
      v[c][i] = live && t + TT * i < P.nz ? cscale(row[c * cs + (t + TT * i) * zs], sc) : mk<C>(0, 0);  // iz < nz <= N/2
  }
  // one twiddle set for the six transforms: forward, and conjugated for the inverse
  C w[E];
  line_twiddles<E, +1>(w, t, P.twz);
#pragma unroll
  for (int c = 0; c < 3; ++c) line_fft_w<E, TT, +1, false, true, S_::PAIR>(v[c], my, t, w);
  if (live) {
    if (P.ipbc == 0) {
      R sxy, sxz, syz;
      zg3_green<N, TT, E>(green_rec(P, kx, ky, 0, sxy, sxz, syz), t, v);
    } else {
#pragma unroll
      for (int i = 0; i < E; ++i) {
        R sxy, sxz, syz;
        C a[6];
        load_rec<T>(green_rec(P, kx, ky, t + TT * i, sxy, sxz, syz), a);
        green_apply(a, sxy, sxz, syz, v[0][i], v[1][i], v[2][i]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) line_fft_w<E, TT, -1, false, false, S_::PAIR, true>(v[c], my, t, w);
  if (live) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const R sc = c == 0 ? sx : (c == 1 ? sy : (R)1);
#pragma unroll
      for (int i = 0; i < H; ++i)
        if (t + TT * i < P.nz) row[c * cs + (t + TT * i) * zs] = cscale(v[c][i], sc);  // keep iz < nz
    }
  }
}

// ZG3R: ZG3 with the block's Green octant lines staged once in shared memory
// and all RHS of the middle-stage batch processed by the same block (IPBC=0,
// five-pass B layout): one L2 read of the octant lines per batch instead of
// one per RHS, and the Green multiply reading shared memory.  Records of 48
// bytes at consecutive kz are read with 16-byte loads at a 48-byte stride,
// free of bank conflicts (3 is odd).
// block: RZ lines x TT threads; grid (ceil(nkx*My/RZ), RHS chunks of zg_rch);
// shared memory: FFT scratch [RZ][lsz] | Green [RZ][N/2+1][6]
template <int N, int TT, int E, typename C>
__device__ __forceinline__ void zg3_green_s(const C* rec, int t, C (&v)[3][E]) {
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int kz = t + TT * i;
    C a[6];
    const float4* g4 = reinterpret_cast<const float4*>(rec + 6 * (kz <= N / 2 ? kz : N - kz));
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const float4 q = g4[m];
      a[2 * m] = mk2<C>(q.x, q.y);
      a[2 * m + 1] = mk2<C>(q.z, q.w);
    }
    if (TT * i + TT - 1 <= N / 2) {
      green_apply_s<1, 1, 1>(a, v[0][i], v[1][i], v[2][i]);
    } else if (TT * i > N / 2) {
      green_apply_s<1, -1, -1>(a, v[0][i], v[1][i], v[2][i]);
    } else {
      if (kz <= N / 2) green_apply_s<1, 1, 1>(a, v[0][i], v[1][i], v[2][i]);
      else green_apply_s<1, -1, -1>(a, v[0][i], v[1][i], v[2][i]);
    }
  }
}

template <typename T, int N> __global__ void __launch_bounds__(128, 3) kx_zg3r(XParams<T> P) {
  using C = cplx<T>;
  using R = T;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RZ = Z3Shape<N>::RZ;
  constexpr int LREC = 6 * (N / 2 + 1);  // complex elements of a line's records
  static_assert(Z3Shape<N>::OK && RZ * TT == 128 && sizeof(C) == 8, "kx_zg3r: FP32, 128-thread blocks");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* my = reinterpret_cast<C*>(smem_raw) + (size_t)l * P.lsz;
  C* gs = reinterpret_cast<C*>(smem_raw) + (size_t)RZ * P.lsz;  // [RZ][N/2+1][6]
  const int nlines = P.nkx * P.My;
  const int p = blockIdx.x * RZ + l;
  const bool live = p < nlines;
  const size_t cs = (size_t)nlines * P.nz;  // component stride of B
  const int kxl = p / P.My;
  const int kx = P.kx0 + kxl, ky = p - kxl * P.My;
  // the block's octant lines: line ll is the contiguous record run of
  // (irx, iry) = (min(kx, Mx - kx), min(ky, My - ky)), kz = 0..N/2
  for (int u = threadIdx.x; u < RZ * (LREC / 2); u += 128) {
    const int ll = u / (LREC / 2), o = u - ll * (LREC / 2);
    const int pp = blockIdx.x * RZ + ll;
    if (pp < nlines) {
      const int kxl2 = pp / P.My, kx2 = P.kx0 + kxl2, ky2 = pp - kxl2 * P.My;
      const int irx = min(kx2, P.Mx - kx2), iry = min(ky2, P.My - ky2);
      const C* src = P.green + ((size_t)irx * (P.My / 2 + 1) + iry) * LREC;
      cp_async16(gs + (size_t)ll * LREC + 2 * o, src + 2 * o);
    }
  }
  const R sx = 2 * kx > P.Mx ? (R)-1 : (R)1, sy = 2 * ky > P.My ? (R)-1 : (R)1;
  C w[E];
  line_twiddles<E, +1>(w, t, P.twz);
  bool staged = false;
  const int rb1 = min(P.nrb_mid, ((int)blockIdx.y + 1) * P.zg_rch);
  for (int rb = (int)blockIdx.y * P.zg_rch; rb < rb1; ++rb) {
    if (xoff(P, P.b_rhs0 + rb)) continue;  // the same for every thread of the block
    C* row = P.B + (size_t)rb * 3 * cs + (size_t)(live ? p : 0) * P.nz;
    C v[3][E];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const R sc = c == 0 ? sx : (c == 1 ? sy : (R)1);
#pragma unroll
      for (int i = 0; i < H; ++i)
        v[c][i] = live && t + TT * i < P.nz ? cscale(row[c * cs + (t + TT * i)], sc) : mk<C>(0, 0);  // iz < nz <= N/2
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) line_fft_w<E, TT, +1, false, true, S_::PAIR>(v[c], my, t, w);
    if (!staged) {
      cp_async_wait_all();
      __syncthreads();  // every thread's Green copies have landed
      staged = true;
    }
    if (live) zg3_green_s<N, TT, E>(gs + (size_t)l * LREC, t, v);
#pragma unroll
    for (int c = 0; c < 3; ++c) line_fft_w<E, TT, -1, false, false, S_::PAIR, true>(v[c], my, t, w);
    if (live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const R sc = c == 0 ? sx : (c == 1 ? sy : (R)1);
#pragma unroll
        for (int i = 0; i < H; ++i)
          if (t + TT * i < P.nz) row[c * cs + (t + TT * i)] = cscale(v[c][i], sc);  // keep iz < nz
      }
    }
  }
  cp_async_wait_all();  // no copy in flight at exit (every RHS masked)
}

// ------------------------------------------------------------- YI: y inverse
// block: RL z-lines x TT; grid (ceil(nz/RL), nkx, 3*nrb)
template <typename T, int N> __global__ void __launch_bounds__(256) kx_yi(const __grid_constant__ XParams<T> P) {
  using C = cplx<T>;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RL = S_::RL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* tile = reinterpret_cast<C*>(smem_raw);
  C* lines = reinterpret_cast<C*>(smem_raw);
  const int iz0 = blockIdx.x * RL, iz = iz0 + l, kxl = blockIdx.y, kx = P.kx0 + kxl;
  const int rb = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3), rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;
  const int nz = P.nz;
  C v[E];
  bool loaded = false;
  if constexpr (tma_rows_ok<N>() && RL == TMA_COLS && sizeof(C) == 8) {
    if (P.tma) {
      // one tensor load of the 256 x 16 tile (z positions beyond n_z read as 0)
      __shared__ __align__(8) uint64_t bar;
      C* tt = tma_tile(smem_raw);
      if (threadIdx.x == 0) mbar_init(&bar, 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar, (N / TMA_ROWS) * TMA_TILE_BYTES);
        tma_load_tile<N>(&P.tmB, tt, iz0, ((rb * 3 + c) * P.nkx + kxl) * P.My, &bar);
      }
      // one decision for the whole block: every thread's bounded wait succeeded
      if (!__syncthreads_and(mbar_wait(&bar, 0, TMA_WAIT_POLLS))) {
        // the copy did not complete in the allowed time: report it, wait once
        // more (bounded) for the copy in flight, and leave this block's lines
        if (threadIdx.x == 0) atomicOr(P.err, 1);
        mbar_wait(&bar, 0, TMA_WAIT_POLLS);
        return;
      }
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = tt[tma_slot(t + TT * i, l)];
      __syncthreads();  // the tile is consumed before the line scratch reuses it
      loaded = true;
    }
  }
  if (!loaded) {
    const C* B = P.B + ((size_t)(rb * 3 + c) * P.nkx + kxl) * (size_t)P.My * nz + iz0;
    load_tile_pairs<RL, N>(B, nz, nz - iz0, tile);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = tile[(t + TT * i) * (RL + 1) + l];
    __syncthreads();  // the tile is consumed before the line scratch reuses it
  }
  line_fft<E, TT, -1, false, false, S_::PAIR>(v, lines + (size_t)l * P.lsy, t, P.twy);
  if (iz < nz) {
    C* A = P.A + (size_t)rl * P.A_rs + ((size_t)(c * nz + iz) * P.Mx + kx) * P.ny;
#pragma unroll
    for (int i = 0; i < H; ++i)
      if (t + TT * i < P.ny) A[t + TT * i] = v[i];  // keep iy < ny
  }
}

// Fused x*y sum of the XI pass: the block total goes to its partial slot; the
// last block of RHS rg (in completion order) folds the nblk partials in a fixed
// order into dot_out[8*rg + dot_k] (deterministic), and the counter wraps to 0.
template <typename T> __device__ __forceinline__ void xdot_reduce(const XParams<T>& P, double2 v, int rg, int blk,
                                                                  int nblk) {
  __shared__ double2 ws[8];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  auto wsum = [](double2 a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a.x += __shfl_down_sync(0xffffffffu, a.x, o);
      a.y += __shfl_down_sync(0xffffffffu, a.y, o);
    }
    return a;
  };
  v = wsum(v);
  if (lane == 0) ws[wid] = v;
  __syncthreads();
  double2* part = P.dot_part + (size_t)rg * nblk;
  if (threadIdx.x == 0) {
    double2 b = make_double2(0.0, 0.0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { b.x += ws[w].x; b.y += ws[w].y; }
    part[blk] = b;
    __threadfence();
    last = atomicInc(P.dot_cnt + rg, (unsigned)nblk - 1) == (unsigned)nblk - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double2 a = make_double2(0.0, 0.0);
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const volatile double* pp = reinterpret_cast<volatile double*>(part + b);
    a.x += pp[0];
    a.y += pp[1];
  }
  a = wsum(a);
  __syncthreads();
  if (lane == 0) ws[wid] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 b = make_double2(0.0, 0.0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { b.x += ws[w].x; b.y += ws[w].y; }
    P.dot_out[(size_t)rg * 8 + P.dot_k] = b;
  }
}

// ------------------------------------------------------------- XI: x inverse + finish
constexpr int XI_STAGE_MAX = 2048;  // largest staged chunk of the XI pass (elements)

// block: RL rows (iy) x TT; grid (ceil(ny/RL), nz, 3*nr)
// shared memory: tile / line scratch [tlx] | x chunk | CXADIA chunk
template <typename T, int N> __global__ void __launch_bounds__(256) kx_xi(const __grid_constant__ XParams<T> P) {
  using C = cplx<T>;
  using S_ = XShape<N>;
  constexpr int E = S_::E, TT = S_::TT, H = S_::H, RL = S_::RL;
  constexpr int MAXC = RL * (N / 2);
  constexpr bool STAGE = MAXC <= XI_STAGE_MAX;  // larger rows keep direct loads (shared memory)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x % TT, l = threadIdx.x / TT;
  C* tile = reinterpret_cast<C*>(smem_raw);
  C* lines = reinterpret_cast<C*>(smem_raw);
  C* xs = reinterpret_cast<C*>(smem_raw) + P.tlx;
  C* as = xs + MAXC;
  const int iy0 = blockIdx.x * RL, iy = iy0 + l, iz = blockIdx.y;
  const int rl = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3);
  if (xoff(P, rl)) return;
  const int ny = P.ny;
  const int S = P.io_full ? P.nat : P.nat0;
  const int SA = P.a_full ? P.nat : P.nat0;
  const C* x = P.x + (size_t)rl * P.x_rs;
  const C* ad = P.adia + (size_t)rl * P.a_rs + (size_t)c * SA;
  // The rows of this block hold one contiguous range of sites (full layout) or
  // of compact indices (compact layout): when x and CXADIA share the layout,
  // both ranges are staged in shared memory together with the A tile, so the
  // finish reads no global memory.
  const int r0 = iy0 + ny * iz, nrows = min(RL, ny - iy0);
  const bool chunked = STAGE && P.io_full == P.a_full;
  int q0 = 0, cnt = 0;
  if (chunked) {
    if (P.io_full) { q0 = P.nx * r0; cnt = nrows * P.nx; }
    else { q0 = P.rowq[r0]; cnt = P.rowq[r0 + nrows] - q0; }
  }
  const int jrow = P.nx * (iy + ny * iz);
  int qi[H];  // x / y index of each kept element, -1 for vacuum
#pragma unroll
  for (int i = 0; i < H; ++i) {
    const int j = jrow + t + TT * i;  // ix < nx
    qi[i] = iy < ny && t + TT * i < P.nx ? (P.io_full ? (P.iocc[j] != 0 ? j : -1) : P.inv[j]) : -1;
  }
  if (chunked) {
    stage_chunk_async<MAXC>(xs, x + (size_t)c * S + q0, cnt);
    stage_chunk_async<MAXC>(as, ad + q0, cnt);
  }
  C v[E];
  bool loaded = false;
  if constexpr (tma_rows_ok<N>() && RL == TMA_COLS && sizeof(C) == 8) {
    if (P.tma_x) {
      // one tensor load of the 256 x 16 tile of A (rows beyond n_y read as 0),
      // while the x and CXADIA chunks arrive by per-thread copies
      __shared__ __align__(8) uint64_t bar;
      C* tt = tma_tile(smem_raw);
      if (threadIdx.x == 0) mbar_init(&bar, 1);
      __syncthreads();
      if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar, (N / TMA_ROWS) * TMA_TILE_BYTES);
        tma_load_tile<N>(&P.tmA, tt, iy0, ((rl * 3 + c) * P.nz + iz) * P.Mx, &bar);
      }
      cp_async_wait_all();  // the x and CXADIA chunks
      // one decision for the whole block (the barrier also publishes every
      // thread's chunk copies): every thread's bounded wait succeeded
      if (!__syncthreads_and(mbar_wait(&bar, 0, TMA_WAIT_POLLS))) {
        // the copy did not complete in the allowed time: report it, wait once
        // more (bounded) for the copy in flight, and leave this block's rows
        if (threadIdx.x == 0) atomicOr(P.err, 1);
        mbar_wait(&bar, 0, TMA_WAIT_POLLS);
        return;
      }
#pragma unroll
      for (int i = 0; i < E; ++i) v[i] = tt[tma_slot(t + TT * i, l)];
      __syncthreads();
      loaded = true;
    }
  }
  if (!loaded) {
    const C* A = P.A + (size_t)rl * P.A_rs + ((size_t)(c * P.nz + iz) * P.Mx) * ny + iy0;
    load_tile_pairs<RL, N>(A, ny, ny - iy0, tile);
    cp_async_wait_all();  // the x and CXADIA chunks
    __syncthreads();
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = tile[(t + TT * i) * (RL + 1) + l];
    __syncthreads();
  }
  line_fft<E, TT, -1, false, false, S_::PAIR>(v, lines + (size_t)l * P.lsx, t, P.twx);
  // finish (cu:116-118): y = CXADIA x - w/ngrid [+ CXAOFF terms], conj for 'C'
  C* y = P.y + (size_t)rl * P.y_rs + (size_t)c * S;
  const C* ao = P.aoff ? P.aoff + (size_t)rl * P.a_rs : nullptr;
  double2 dacc = make_double2(0.0, 0.0);  // x*y of this thread's sites (dot_out)
#pragma unroll
  for (int i = 0; i < H; ++i) {
    if (iy >= ny) break;
    if (t + TT * i >= P.nx) continue;  // padded FFT length: ix beyond the row
    const int j = jrow + t + TT * i;
    const int q = qi[i];
    if (q < 0) {
      if (P.io_full) y[j] = mk<C>(0, 0);
      continue;
    }
    int qa = q;
    if (!chunked) qa = P.a_full ? j : P.inv[j];
    C xc = chunked ? xs[q - q0] : x[(size_t)c * S + q];
    const C av = chunked ? as[q - q0] : ad[qa];
    if (P.conj) xc.y = -xc.y;
    C yv = csub(cmul(av, xc), cscale(v[i], P.inv_ngrid));
    if (ao) {
      C x1 = x[q], x2 = x[S + q], x3 = x[2 * (size_t)S + q];
      if (P.conj) { x1.y = -x1.y; x2.y = -x2.y; x3.y = -x3.y; }
      const C a23 = ao[qa], a31 = ao[SA + qa], a12 = ao[2 * (size_t)SA + qa];
      if (c == 0) yv = cadd(yv, cadd(cmul(a31, x3), cmul(a12, x2)));
      else if (c == 1) yv = cadd(yv, cadd(cmul(a12, x1), cmul(a23, x3)));
      else yv = cadd(yv, cadd(cmul(a23, x2), cmul(a31, x1)));
    }
    if (P.conj) yv.y = -yv.y;
    y[q] = yv;
    if (P.dot_out) {  // conj = 0 here: xc is x
      const double2 xd = to_d(xc), yd = to_d(yv);
      dacc.x += xd.x * yd.x - xd.y * yd.y;
      dacc.y += xd.x * yd.y + xd.y * yd.x;
    }
  }
  if (P.dot_out)
    xdot_reduce(P, dacc, P.rhs0 + rl, (c * (int)gridDim.y + (int)blockIdx.y) * (int)gridDim.x + (int)blockIdx.x,
                3 * (int)gridDim.y * (int)gridDim.x);
}

// ------------------------------------------------------------- XYF / XYI: fused xy passes of a z plane
// One cluster of four CTAs per (RHS, component, iz).  The plane of the
// x-transformed rows, ny x M_x complex (256 KB at 128 x 256), is spread over
// the four CTAs' shared memory by kx mod 4: CTA q holds the columns
// kx = 4m + q as [iy][m] with the odd row stride M_x/4 + 1, so that column
// reads are free of bank conflicts.  A row transform's thread t owns the
// outputs kx = t + TX*i (line_fft), all in the plane of CTA t % 4.
//   XYF: CTA q transforms rows iy in [q*rpc, (q+1)*rpc) along x and stores
//        the outputs in the owning planes (distributed shared memory); after
//        the cluster barrier each CTA transforms its M_x/4 columns along y
//        and writes B[c][kx][iz][ky] (ky contiguous, coalesced from
//        registers).
//   XYI: each CTA reads its columns of B, transforms them back along y
//        keeping iy < ny into its plane; after the cluster barrier CTA q
//        reads rows iy in [q*rpc, (q+1)*rpc) from the four planes, transforms
//        them back along x keeping ix < nx and finishes as the XI pass does.
// Peer shared memory is touched only between cluster barriers that every
// thread of the four CTAs reaches (the CTAs of a cluster share RHS,
// component and iz, so a masked RHS returns in all four before the first).
template <int NX, int NY> struct XYShape {
  static constexpr int EX = RegShape<NX>::E, TX = RegShape<NX>::T, HX = EX / 2, RX = 256 / TX;
  static constexpr int EY = RegShape<NY>::E, TY = RegShape<NY>::T, HY = EY / 2, CY = 256 / TY;
  static constexpr int MQ = NX / 4;                    // plane columns per CTA
  static constexpr int PR = NY / 2;                    // plane rows (ny <= NY/2)
  static constexpr int PS = MQ + 1;                    // plane row stride (odd)
  static constexpr int PLANE = (PR * PS + 1) / 2 * 2;  // elements; even, so the scratch after it is 16-byte aligned
  static constexpr bool OK = TX % 4 == 0 && MQ % 2 == 0;
};

template <int NX, int NY> __global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(256, 2) kxy_f(XParams<float> P) {
  using C = float2;
  using S = XYShape<NX, NY>;
  constexpr int EX = S::EX, TX = S::TX, HX = S::HX, RX = S::RX;
  constexpr int EY = S::EY, TY = S::TY, HY = S::HY, CY = S::CY, MQ = S::MQ, PS = S::PS;
  static_assert(S::OK, "row outputs of one thread must share kx mod 4");
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* plane = reinterpret_cast<C*>(smem_raw);  // [PR][PS]
  C* lines = plane + S::PLANE;                // row / column FFT scratch
  const int q = (int)cl.block_rank();
  const int iz = blockIdx.y, rb = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3), rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;  // all four CTAs of the cluster
  const int nx = P.nx, ny = P.ny;
  const int rpc = (ny + 3) / 4, row0 = q * rpc, row1 = min(ny, row0 + rpc);
  {
    const int t = threadIdx.x % TX, l = threadIdx.x / TX;
    C* dst = cl.map_shared_rank(plane, t & 3);  // kx = t + TX*i: kx % 4 = t % 4
    C* ln = lines + (size_t)l * P.lsx;
    const int S_ = P.io_full ? P.nat : P.nat0;
    const C* x = P.x + (size_t)rl * P.x_rs + (size_t)c * S_;
    cl.sync();  // every CTA of the cluster runs before a peer writes its plane
    for (int r0 = row0; r0 < row1; r0 += RX) {
      const int iy = r0 + l;
      const bool live = iy < row1;
      const int jrow = nx * (iy + ny * iz);
      C v[EX];
      if (P.io_full) {
#pragma unroll
        for (int i = 0; i < HX; ++i) v[i] = live && t + TX * i < nx ? x[jrow + t + TX * i] : mk<C>(0, 0);
      } else {
        int qi[HX];
#pragma unroll
        for (int i = 0; i < HX; ++i) qi[i] = live && t + TX * i < nx ? P.inv[jrow + t + TX * i] : -1;
#pragma unroll
        for (int i = 0; i < HX; ++i) v[i] = qi[i] >= 0 ? x[qi[i]] : mk<C>(0, 0);
      }
      if (P.conj) {
#pragma unroll
        for (int i = 0; i < HX; ++i) v[i].y = -v[i].y;
      }
      line_fft<EX, TX, +1, false, true, XShape<NX>::PAIR>(v, ln, t, P.twx);
      if (live) {
#pragma unroll
        for (int i = 0; i < EX; ++i) dst[iy * PS + (t >> 2) + (TX / 4) * i] = v[i];
      }
    }
  }
  cl.sync();  // the four planes are complete (and the row scratch is free)
  {
    const int t = threadIdx.x % TY, l = threadIdx.x / TY;
    C* ln = lines + (size_t)l * P.lsy;
    const size_t cs = (size_t)NX * P.nz * NY;  // component stride of B
    C* Bc = P.B + (size_t)(rb * 3 + c) * cs + (size_t)iz * NY;
    for (int m0 = 0; m0 < MQ; m0 += CY) {
      const int m = m0 + l;
      const bool live = m < MQ;
      C v[EY];
#pragma unroll
      for (int i = 0; i < HY; ++i) v[i] = live && t + TY * i < ny ? plane[(t + TY * i) * PS + m] : mk<C>(0, 0);
      line_fft<EY, TY, +1, false, true, XShape<NY>::PAIR>(v, ln, t, P.twy);
      if (live) {
        C* b = Bc + (size_t)(4 * m + q) * P.nz * NY;
#pragma unroll
        for (int i = 0; i < EY; ++i) b[t + TY * i] = v[i];
      }
    }
  }
}

template <int NX, int NY> __global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(256, 2) kxy_i(XParams<float> P) {
  using C = float2;
  using S = XYShape<NX, NY>;
  constexpr int EX = S::EX, TX = S::TX, HX = S::HX, RX = S::RX;
  constexpr int EY = S::EY, TY = S::TY, HY = S::HY, CY = S::CY, MQ = S::MQ, PS = S::PS;
  static_assert(S::OK, "row inputs of one thread must share kx mod 4");
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* plane = reinterpret_cast<C*>(smem_raw);
  C* lines = plane + S::PLANE;
  const int q = (int)cl.block_rank();
  const int iz = blockIdx.y, rb = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3), rl = P.b_rhs0 + rb;
  if (xoff(P, rl)) return;  // all four CTAs of the cluster
  const int nx = P.nx, ny = P.ny;
  {
    const int t = threadIdx.x % TY, l = threadIdx.x / TY;
    C* ln = lines + (size_t)l * P.lsy;
    const size_t cs = (size_t)NX * P.nz * NY;
    const C* Bc = P.B + (size_t)(rb * 3 + c) * cs + (size_t)iz * NY;
    for (int m0 = 0; m0 < MQ; m0 += CY) {
      const int m = m0 + l;
      const bool live = m < MQ;
      const C* b = Bc + (size_t)(4 * (live ? m : 0) + q) * P.nz * NY;
      C v[EY];
#pragma unroll
      for (int i = 0; i < EY; ++i) v[i] = live ? b[t + TY * i] : mk<C>(0, 0);
      line_fft<EY, TY, -1, false, false, XShape<NY>::PAIR>(v, ln, t, P.twy);
      if (live) {
#pragma unroll
        for (int i = 0; i < HY; ++i)
          if (t + TY * i < ny) plane[(t + TY * i) * PS + m] = v[i];  // keep iy < ny
      }
    }
  }
  cl.sync();  // the four planes are complete (and the column scratch is free)
  double2 dacc = make_double2(0.0, 0.0);  // x*y of this thread's sites (dot_out)
  {
    const int t = threadIdx.x % TX, l = threadIdx.x / TX;
    const C* src = cl.map_shared_rank(plane, t & 3);
    C* ln = lines + (size_t)l * P.lsx;
    const int rpc = (ny + 3) / 4, row0 = q * rpc, row1 = min(ny, row0 + rpc);
    const int S_ = P.io_full ? P.nat : P.nat0;
    const int SA = P.a_full ? P.nat : P.nat0;
    const C* x = P.x + (size_t)rl * P.x_rs;
    const C* ad = P.adia + (size_t)rl * P.a_rs + (size_t)c * SA;
    C* y = P.y + (size_t)rl * P.y_rs + (size_t)c * S_;
    const C* ao = P.aoff ? P.aoff + (size_t)rl * P.a_rs : nullptr;
    for (int r0 = row0; r0 < row1; r0 += RX) {
      const int iy = r0 + l;
      const bool live = iy < row1;
      const int jrow = nx * (iy + ny * iz);
      int qi[HX];  // x / y index of each kept element, -1 for vacuum
#pragma unroll
      for (int i = 0; i < HX; ++i) {
        const int j = jrow + t + TX * i;
        qi[i] = live && t + TX * i < nx ? (P.io_full ? (P.iocc[j] != 0 ? j : -1) : P.inv[j]) : -1;
      }
      C v[EX];
#pragma unroll
      for (int i = 0; i < EX; ++i) v[i] = live ? src[iy * PS + (t >> 2) + (TX / 4) * i] : mk<C>(0, 0);
      line_fft<EX, TX, -1, false, false, XShape<NX>::PAIR>(v, ln, t, P.twx);
      // finish (cu:116-118): y = CXADIA x - w/ngrid [+ CXAOFF terms], conj for 'C'
#pragma unroll
      for (int i = 0; i < HX; ++i) {
        if (!live || t + TX * i >= nx) continue;
        const int j = jrow + t + TX * i;
        const int qx = qi[i];
        if (qx < 0) {
          if (P.io_full) y[j] = mk<C>(0, 0);
          continue;
        }
        const int qa = P.a_full == P.io_full ? qx : (P.a_full ? j : P.inv[j]);
        C xc = x[(size_t)c * S_ + qx];
        if (P.conj) xc.y = -xc.y;
        C yv = csub(cmul(ad[qa], xc), cscale(v[i], P.inv_ngrid));
        if (ao) {
          C x1 = x[qx], x2 = x[S_ + qx], x3 = x[2 * (size_t)S_ + qx];
          if (P.conj) { x1.y = -x1.y; x2.y = -x2.y; x3.y = -x3.y; }
          const C a23 = ao[qa], a31 = ao[SA + qa], a12 = ao[2 * (size_t)SA + qa];
          if (c == 0) yv = cadd(yv, cadd(cmul(a31, x3), cmul(a12, x2)));
          else if (c == 1) yv = cadd(yv, cadd(cmul(a12, x1), cmul(a23, x3)));
          else yv = cadd(yv, cadd(cmul(a23, x2), cmul(a31, x1)));
        }
        if (P.conj) yv.y = -yv.y;
        y[qx] = yv;
        if (P.dot_out) {  // conj = 0 here: xc is x
          const double2 xd = to_d(xc), yd = to_d(yv);
          dacc.x += xd.x * yd.x - xd.y * yd.y;
          dacc.y += xd.x * yd.y + xd.y * yd.x;
        }
      }
    }
  }
  cl.sync();  // no CTA leaves while a peer still reads its plane
  if (P.dot_out) xdot_reduce(P, dacc, P.rhs0 + rl, (c * P.nz + iz) * 4 + q, 12 * P.nz);
}

// ------------------------------------------------------------- host side
// ZGT / ZG3T: the z passes on the B layout of the fused xy passes
enum class XPass { XF, YF, ZG, ZG3, YI, XI, ZGT, ZG3T, ZG3R };

// z passes on the B layout of the fused xy passes (z stride M_y = BTY)
template <typename T, int N, int BTY> static const void* xkt(XPass p) {
  if constexpr (sizeof(T) == 4) {
    if (p == XPass::ZGT) return (const void*)kx_zg<T, N, BTY>;
    if constexpr (Z3Shape<N>::OK)
      if (p == XPass::ZG3T) return (const void*)kx_zg3<T, N, BTY>;
  }
  return nullptr;
}

template <typename T, int N> static const void* xk(XPass p, int my = 0) {
  if (p == XPass::ZGT || p == XPass::ZG3T) {
    switch (my) {
      case 64: return xkt<T, N, 64>(p);
      case 128: return xkt<T, N, 128>(p);
      case 256: return xkt<T, N, 256>(p);
      default: return nullptr;
    }
  }
  switch (p) {
    case XPass::XF: return (const void*)kx_xf<T, N>;
    case XPass::YF: return (const void*)kx_yf<T, N>;
    case XPass::ZG: return (const void*)kx_zg<T, N>;
    case XPass::ZG3:
      if constexpr (Z3Shape<N>::OK && sizeof(T) == 4) return (const void*)kx_zg3<T, N>;
      return nullptr;
    case XPass::ZG3R:
      if constexpr (Z3Shape<N>::OK && sizeof(T) == 4 && 128 / RegShape<N>::T * RegShape<N>::T == 128)
        return (const void*)kx_zg3r<T, N>;
      return nullptr;

    case XPass::YI: return (const void*)kx_yi<T, N>;
    default: return (const void*)kx_xi<T, N>;
  }
}

// my: M_y, for the z passes on the fused layout (ZGT, ZG3T)
template <typename T> static const void* xkernel(XPass p, int n, int my = 0) {
  switch (n) {
    case 16: return xk<T, 16>(p, my);
    case 32: return xk<T, 32>(p, my);
    case 48: return xk<T, 48>(p, my);
    case 64: return xk<T, 64>(p, my);
    case 96: return xk<T, 96>(p, my);
    case 128: return xk<T, 128>(p, my);
    case 192: return xk<T, 192>(p, my);
    case 256: return xk<T, 256>(p, my);
    case 512:
      if constexpr (sizeof(T) == 4) return xk<T, 512>(p, my);  // FP64: shared memory of the 512 passes too large
      return nullptr;
    default: return nullptr;
  }
}

static int rT(int n) { return reg_threads(n); }

// fused xy kernels for (M_x, M_y); nullptr where none is built
static const void* xykernel(bool fwd, int nxl, int nyl) {
#define DDB_XY(a, b) \
  if (nxl == a && nyl == b) return fwd ? (const void*)kxy_f<a, b> : (const void*)kxy_i<a, b>;
  DDB_XY(64, 64) DDB_XY(128, 128) DDB_XY(256, 256) DDB_XY(128, 256) DDB_XY(256, 128)
#undef DDB_XY
  return nullptr;
}
// shared memory of kxy_f / kxy_i: plane (XYShape::PLANE) + row or column FFT scratch
static size_t xy_smem(int nxl, int nyl, int lsx, int lsy) {
  const int TX = reg_threads(nxl), TY = reg_threads(nyl);
  const int PS = nxl / 4 + 1, PLANE = ((nyl / 2) * PS + 1) / 2 * 2;
  return ((size_t)PLANE + std::max((size_t)(256 / TX) * lsx, (size_t)(256 / TY) * lsy)) * sizeof(float2);
}

template <typename T> static int xlaunch(const void* f, dim3 g, int th, size_t sm, cudaStream_t st, XParams<T>& P) {
  raise_smem_limit(f);
  void* args[] = {(void*)&P};
  note_launch();
  cudaError_t e = cudaLaunchKernel(f, g, dim3(th), args, sm, st);
  if (e != cudaSuccess) { set_cuda_error("MATVEC launch", e); return 1; }
  return 0;
}

bool xzg3_supported(int Mz) { return xkernel<float>(XPass::ZG3, Mz) != nullptr; }

template <typename T> bool xpipe_supported(const Geometry& g) {
  if (env_flag("DDSCAT_B200_ZFIRST")) return false;
  // FP64: axis lengths up to 256 (the shared memory of the 512-point passes is too large in complex double)
  auto ok = [](int n) { return xreg_supported(n) && (sizeof(T) == 4 || n <= 256); };
  return ok(g.Mx) && ok(g.My) && ok(g.Mz);
}

// cuTensorMapEncodeTiled of the driver, looked up once through the runtime
// (no link against the driver library)
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// Map of B (rows of n_z complex floats, row stride n_z * 8 bytes) for the
// 256-point y passes' tiles, or of A (rows of n_y) for the x passes: box
// {16, 256}, 128-byte swizzle, zero fill.
static bool encode_b_map(CUtensorMap* m, void* base, size_t rows, int nz) {
  const auto enc = tensor_map_encoder();
  if (!enc || rows > 0xffffffffull || (nz & 1)) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)nz, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)nz * 8};
  const cuuint32_t box[2] = {(cuuint32_t)TMA_COLS, (cuuint32_t)TMA_ROWS};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T> int matvec_check(Engine<T>& E) {
  if (!E.d_err) return 0;
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, E.d_err, sizeof(int), cudaMemcpyDeviceToHost, E.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(E.stream);
  if (e != cudaSuccess) { set_cuda_error("MATVEC status", e); return 26; }
  if (h == 0) return 0;
  cudaMemsetAsync(E.d_err, 0, sizeof(int), E.stream);
  set_error("MATVEC", "a tile copy of the y passes did not complete in the allowed time");
  return 26;
}
template int matvec_check<float>(Engine<float>&);
template int matvec_check<double>(Engine<double>&);

template <typename T>
int matvec_xpipe(Engine<T>& E, const MvArgs<T>& a) {
  using C = cplx<T>;
  const Geometry& g = E.g;
  XParams<T> P{};
  P.err = E.d_err;
  P.nx = g.nx; P.ny = g.ny; P.nz = g.nz; P.Mx = g.Mx; P.My = g.My; P.Mz = g.Mz;
  P.nat = g.nat; P.nat0 = g.nat0;
  P.x_rs = a.x_rs; P.y_rs = a.y_rs; P.a_rs = a.a_rs;
  P.io_full = a.io_full; P.a_full = a.a_full; P.conj = a.conj;
  P.inv = E.inv; P.iocc = E.iocc; P.rowq = E.rowq; P.mask = a.mask;
  P.A = E.zhat; P.A_rs = (size_t)3 * g.nz * g.Mx * g.ny;
  P.B = E.slab;
  P.green = E.green; P.ipbc = g.ipbc;
  P.twx = E.twx; P.twy = E.twy; P.twz = E.twz;
  P.inv_ngrid = (T)(1.0 / (double)g.ngrid());
  P.dot_out = a.dot_out; P.dot_part = a.dot_part; P.dot_cnt = a.dot_cnt; P.dot_k = a.dot_k;
  if (a.dot_out && (a.conj || !a.dot_part || !a.dot_cnt)) { set_error("MATVEC", "fused x*y sum needs conj = 0"); return 25; }
  const int TX = rT(g.Mx), TY = rT(g.My), TZ = rT(g.Mz);
  const int RX = 256 / TX, RY = 256 / TY;
  const int RZ = std::max(1, 128 / TZ);  // ZG: 3*TZ*RZ threads
  // ZG3 (components in registers, E <= 16) unless the engine's tunable (autotuner
  // or DDSCAT_B200_ZG=1) selects ZG
  const void* fzg3 = E.tune_zg ? nullptr : xkernel<T>(XPass::ZG3, g.Mz);
  const int RZ3 = 128 / TZ;  // ZG3: RZ3 lines of TZ threads
  // must match XShape<N>::PAIR
  P.lsx = line_stride(g.Mx / TX, TX, RX, false, TX >= 8);
  P.lsy = line_stride(g.My / TY, TY, RY, false, TY >= 8);
  P.lsz = fzg3 ? line_stride(g.Mz / TZ, TZ, RZ3, false, TZ >= 8)
               : std::max(line_stride(g.Mz / TZ, TZ, RZ, false, TZ >= 8), g.Mz);
  // the transpose tile and the line scratch share one region
  P.tlx = (int)std::max((size_t)g.Mx * (RX + 1), (size_t)RX * P.lsx);
  // a tensor tile of the x passes (32 KB at a 1024-byte boundary) fits in front of the XI chunks
  if (g.Mx == 256 || g.Mx == 512)
    P.tlx = std::max(P.tlx, (int)(((size_t)(g.Mx / TMA_ROWS) * TMA_TILE_BYTES + 1024) / sizeof(C)));
  const size_t smx = (size_t)P.tlx * sizeof(C);
  // XI: the x and CXADIA chunks of RX rows, each sized as the kernel lays them
  // out (MAXC = RL * N/2 elements, which is RX * nx only when Mx = 2 nx)
  const size_t xi_maxc = (size_t)RX * (g.Mx / 2);
  const size_t smxi = smx + (xi_maxc <= (size_t)XI_STAGE_MAX ? 2 * xi_maxc * sizeof(C) : 0);
  size_t smy = std::max((size_t)g.My * (RY + 1), (size_t)RY * P.lsy) * sizeof(C);
  // tensor tiles for the 256-point y passes (FP32, five-pass B layout): the
  // slab as rows of n_z; the tile needs 32 KB at a 1024-byte boundary
  P.tma = 0;
  P.tma_x = 0;
  if constexpr (sizeof(T) == 4) {
    // the same for A (rows of n_y) in the 256-point x passes
    if (E.use_tma && (g.Mx == 256 || g.Mx == 512) && RX == TMA_COLS && E.d_err &&
        encode_b_map(&P.tmA, E.zhat, (size_t)E.zcap * 3 * g.nz * g.Mx, g.ny))
      P.tma_x = 1;
    if (E.use_tma && (g.My == 256 || g.My == 512) && RY == TMA_COLS && E.d_err &&
        encode_b_map(&P.tmB, E.slab, (size_t)E.slab_nr * 3 * E.slab_B * g.My, g.nz)) {
      P.tma = 1;
      smy = std::max(smy, (size_t)(g.My / TMA_ROWS) * TMA_TILE_BYTES + 1024);
    }
  }
  // ZG3: FFT scratch
  const size_t smz = fzg3 ? (size_t)RZ3 * P.lsz * sizeof(C) : (size_t)3 * RZ * P.lsz * sizeof(C);
  // ZG3R (Green lines staged once per block and reused for a chunk of RHS):
  // IPBC=0, batches of at least 4 RHS (DDSCAT_B200_NOZG3R=1 keeps ZG3)
  const void* fzg3r = fzg3 && g.ipbc == 0 && !env_flag("DDSCAT_B200_NOZG3R") ? xkernel<T>(XPass::ZG3R, g.Mz) : nullptr;
  const size_t smzr = smz + (size_t)RZ3 * 6 * (g.Mz / 2 + 1) * sizeof(C);
  const void* fxf = xkernel<T>(XPass::XF, g.Mx);
  const void* fyf = xkernel<T>(XPass::YF, g.My);
  const void* fzg = xkernel<T>(XPass::ZG, g.Mz);
  const void* fyi = xkernel<T>(XPass::YI, g.My);
  const void* fxi = xkernel<T>(XPass::XI, g.Mx);
  // DDSCAT_B200_FUSEXY=1, FP32 with all kx planes of a slab batch resident
  // (FFT3D): the x and y passes fused per z plane (kxy_f / kxy_i), three
  // launches per slab batch.  Opt-in: at 128^3 it moves 41 % fewer DRAM bytes
  // in the xy passes but runs slower than the five-pass schedule (16 warps per
  // SM at 101 KB of shared memory per CTA, and half-used sectors in the z
  // pass on the ky-contiguous layout).
  const void* fxyf = nullptr;
  const void* fxyi = nullptr;
  if constexpr (sizeof(T) == 4) {
    if (E.slab_B == g.Mx && env_flag("DDSCAT_B200_FUSEXY")) {
      fxyf = xykernel(true, g.Mx, g.My);
      fxyi = xykernel(false, g.Mx, g.My);
    }
  }
  const void* fzt = fxyf ? xkernel<T>(fzg3 ? XPass::ZG3T : XPass::ZGT, g.Mz, g.My) : nullptr;
  if (fxyf && fxyi && fzt) {
    const size_t smxy = xy_smem(g.Mx, g.My, P.lsx, P.lsy);
    P.kx0 = 0;
    P.nkx = g.Mx;
    P.b_rhs0 = 0;
    for (int r0 = 0; r0 < a.nrhs; r0 += E.slab_nr) {
      const int nr = std::min(E.slab_nr, a.nrhs - r0);
      P.rhs0 = r0;
      P.x = a.x + (size_t)r0 * a.x_rs;
      P.y = a.y + (size_t)r0 * a.y_rs;
      P.adia = a.adia + (size_t)r0 * a.a_rs;
      P.aoff = a.aoff ? a.aoff + (size_t)r0 * a.a_rs : nullptr;
      const dim3 gxy(4u, (unsigned)g.nz, (unsigned)(3 * nr));
      if (xlaunch<T>(fxyf, gxy, 256, smxy, E.stream, P)) return 21;
      if (fzg3 ? xlaunch<T>(fzt, dim3((unsigned)nr, (unsigned)ceil_div((size_t)g.Mx * g.My, RZ3)), 128, smz,
                            E.stream, P)
               : xlaunch<T>(fzt, dim3((unsigned)nr, (unsigned)ceil_div((size_t)g.Mx * g.My, RZ)), 3 * TZ * RZ, smz,
                            E.stream, P))
        return 23;
      if (xlaunch<T>(fxyi, gxy, 256, smxy, E.stream, P)) return 25;
    }
    return 0;
  }
  for (int r0 = 0; r0 < a.nrhs; r0 += E.zcap) {
    const int nr = std::min(E.zcap, a.nrhs - r0);
    P.rhs0 = r0;
    P.x = a.x + (size_t)r0 * a.x_rs;
    P.y = a.y + (size_t)r0 * a.y_rs;
    P.adia = a.adia + (size_t)r0 * a.a_rs;
    P.aoff = a.aoff ? a.aoff + (size_t)r0 * a.a_rs : nullptr;
    if (xlaunch<T>(fxf, dim3((unsigned)ceil_div(g.ny, RX), (unsigned)g.nz, (unsigned)(3 * nr)), 256, smx, E.stream, P))
      return 21;
    for (int rb0 = 0; rb0 < nr; rb0 += E.slab_nr) {
      const int nrb = std::min(E.slab_nr, nr - rb0);
      P.b_rhs0 = rb0;
      P.nrb_mid = nrb;
      for (int kx0 = 0; kx0 < g.Mx; kx0 += E.slab_B) {
        P.kx0 = kx0;
        P.nkx = std::min(E.slab_B, g.Mx - kx0);
        if (xlaunch<T>(fyf, dim3((unsigned)ceil_div(g.nz, RY), (unsigned)P.nkx, (unsigned)(3 * nrb)), 256, smy,
                       E.stream, P))
          return 22;
        // ZG3R: RHS chunks so that the grid has at least 4 waves of 3 blocks per SM
        const size_t nlb = ceil_div((size_t)P.nkx * g.My, RZ3);
        const int nchunk = (int)std::min<size_t>((size_t)nrb, std::max<size_t>(1, ceil_div(4 * 3 * 148, nlb)));
        P.zg_rch = (int)ceil_div((size_t)nrb, (size_t)nchunk);
        const bool use_r = fzg3r && P.zg_rch >= E.zg3r_min;
        if (use_r ? xlaunch<T>(fzg3r, dim3((unsigned)nlb, (unsigned)ceil_div((size_t)nrb, (size_t)P.zg_rch)), 128, smzr,
                               E.stream, P)
            : fzg3 ? xlaunch<T>(fzg3, dim3((unsigned)nrb, (unsigned)ceil_div((size_t)P.nkx * g.My, RZ3)), 128, smz,
                              E.stream, P)
                 : xlaunch<T>(fzg, dim3((unsigned)nrb, (unsigned)ceil_div((size_t)P.nkx * g.My, RZ)), 3 * TZ * RZ,
                              smz, E.stream, P))
          return 23;
        if (xlaunch<T>(fyi, dim3((unsigned)ceil_div(g.nz, RY), (unsigned)P.nkx, (unsigned)(3 * nrb)), 256, smy,
                       E.stream, P))
          return 24;
      }
    }
    if (xlaunch<T>(fxi, dim3((unsigned)ceil_div(g.ny, RX), (unsigned)g.nz, (unsigned)(3 * nr)), 256, smxi, E.stream, P))
      return 25;
  }
  return 0;
}

// partial sums per RHS of the fused x*y sum: XI blocks, or the 4 CTAs per
// (component, iz) of the fused XYI pass
size_t xdot_blocks(const Geometry& g) {
  return std::max((size_t)3 * g.nz * ceil_div(g.ny, 256 / reg_threads(g.Mx)), (size_t)12 * g.nz);
}

// planar [6][Z][Y][X] (build / CXZC layout) -> [X][Y][Z][6]
template <typename C> __global__ void k_interleave6_zfast(const C* src, C* dst, int X, int Y, int Z) {
  const size_t npts = (size_t)X * Y * Z;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 6 * npts; i += (size_t)gridDim.x * blockDim.x) {
    const size_t m = i / npts, p = i - m * npts;
    const size_t ix = p % X, iy = (p / X) % Y, iz = p / ((size_t)X * Y);
    dst[((ix * Y + iy) * Z + iz) * 6 + m] = src[i];
  }
}

template <typename T> int interleave_green_zfast(Engine<T>& E, const cplx<T>* planar) {
  const Geometry& g = E.g;
  const int X = g.ipbc == 0 ? g.Mx / 2 + 1 : g.Mx, Y = g.ipbc == 0 ? g.My / 2 + 1 : g.My,
            Z = g.ipbc == 0 ? g.Mz / 2 + 1 : g.Mz;
  const size_t n = (size_t)6 * X * Y * Z;
  k_interleave6_zfast<cplx<T>><<<(unsigned)std::min<size_t>(ceil_div(n, 256), 148 * 32), 256, 0, E.stream>>>(
      planar, E.green, X, Y, Z);
  note_launch();
  return check_launch("Green interleave (z-fastest)");
}

template <typename T> int xpipe_len(int m) {
  for (int L : {16, 32, 48, 64, 96, 128, 192, 256, 512})
    if (L >= m && xreg_supported(L) && (sizeof(T) == 4 || L <= 256)) return L;
  return 0;
}

template int xpipe_len<float>(int);
template int xpipe_len<double>(int);
template bool xpipe_supported<float>(const Geometry&);
template bool xpipe_supported<double>(const Geometry&);
template int matvec_xpipe<float>(Engine<float>&, const MvArgs<float>&);
template int matvec_xpipe<double>(Engine<double>&, const MvArgs<double>&);
template int interleave_green_zfast<float>(Engine<float>&, const float2*);
template int interleave_green_zfast<double>(Engine<double>&, const double2*);

}  // namespace ddb
