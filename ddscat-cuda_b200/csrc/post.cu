// EVALQ and far-field (SCAT) kernels (sm_100a).
//
// EVALQ restates ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu:770-783 and
// :939-950: q = (CXADIA + i (2/3) k^3) P + CXAOFF block terms, then FP64
// products P^H q and E^H P.
//
// The far-field sums S_d = sum_j P_j exp(-i k_d . r_j), r_j = ((i+1)+x0)*dx
// (cu:793-822), are evaluated with a separable phase: exp(-i k.r) =
// ex_d[ix] * ey_d[iy] * ez_d[iz], three 1-D tables per direction built in FP64,
// so each dipole-direction term costs two complex multiplies instead of a
// sincosf.  A block keeps DIRS directions in shared memory and reads each
// dipole's polarisation once for all of them; partial sums are combined in a
// fixed order (deterministic).
#include <algorithm>
#include <vector>
#include "solvers.h"

namespace ddb {

template <typename C>
__global__ void k_evalq_q(const C* p, C* q, const C* ad, const C* ao, const int* occ, int nat, int nat0, int a_full,
                          double rabs_im) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nat0) return;
  const size_t jf = a_full ? (size_t)occ[j] : (size_t)j;
  const size_t st = a_full ? (size_t)nat : (size_t)nat0;
  const C p1 = p[j], p2 = p[j + nat0], p3 = p[j + 2 * (size_t)nat0];
  C d1 = ad[jf], d2 = ad[jf + st], d3 = ad[jf + 2 * st];
  const float ri = (float)rabs_im;  // the reference stores i*(2/3)k^3 as a float
  d1.y += ri; d2.y += ri; d3.y += ri;
  C q1 = cmul(d1, p1), q2 = cmul(d2, p2), q3 = cmul(d3, p3);
  if (ao) {
    const C a23 = ao[jf], a31 = ao[jf + st], a12 = ao[jf + 2 * st];
    q1 = cadd(q1, cadd(cmul(a31, p3), cmul(a12, p2)));
    q2 = cadd(q2, cadd(cmul(a12, p1), cmul(a23, p3)));
    q3 = cadd(q3, cadd(cmul(a23, p2), cmul(a31, p1)));
  }
  q[j] = q1;
  q[j + nat0] = q2;
  q[j + 2 * (size_t)nat0] = q3;
}

template <typename T>
int evalq_compute(Engine<T>& eng, VecOps<T>& ops, const cplx<T>* e, const cplx<T>* p, const cplx<T>* adia,
                  const cplx<T>* aoff, int a_full, cplx<T>* qbuf, double ak3, double2* zabs, double2* zep) {
  const int nat0 = eng.g.nat0;
  k_evalq_q<<<(unsigned)ceil_div(nat0, 256), 256, 0, ops.stream>>>(p, qbuf, adia, aoff, eng.occ, eng.g.nat, nat0, a_full,
                                                                   ak3 / 1.5);
  note_launch();
  if (check_launch("GPU EVALQ local alpha^-1 P")) return 306;
  const cplx<T>* A[2] = {p, e};
  const cplx<T>* B[2] = {qbuf, p};
  const int cj[2] = {1, 1};
  double2 o[2];
  if (ops.dots(3 * nat0, 2, A, B, cj, o)) return 307;
  *zabs = o[0];
  *zep = o[1];
  return 0;
}

// ---------------------------------------------------------------- far field
constexpr int FF_THREADS = 256;
constexpr int FF_DIRS = 8;

// tables[d][0..nx) = exp(-i kx (ix+1+x0x) dx), then ny, then nz entries
__global__ void k_ff_tables(const double* dirs, int ndir, int nx, int ny, int nz, double dx0, double dx1, double dx2,
                            double x00, double x01, double x02, float2* tab) {
  const int ntab = nx + ny + nz;
  const size_t tot = (size_t)ndir * ntab;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot; t += (size_t)gridDim.x * blockDim.x) {
    const int d = (int)(t / ntab), u = (int)(t % ntab);
    double ph;
    if (u < nx) ph = dirs[3 * d] * ((u + 1) + x00) * dx0;
    else if (u < nx + ny) ph = dirs[3 * d + 1] * ((u - nx + 1) + x01) * dx1;
    else ph = dirs[3 * d + 2] * ((u - nx - ny + 1) + x02) * dx2;
    double s, c;
    sincos(ph, &s, &c);
    tab[t] = make_float2((float)c, (float)-s);
  }
}

__global__ void k_pack_coords(const int* occ, int nat0, int nx, int ny, unsigned* packed) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nat0) return;
  const int j = occ[q];
  const unsigned ix = j % nx, iy = (j / nx) % ny, iz = j / (nx * ny);
  packed[q] = ix | (iy << 11) | (iz << 22);
}

template <typename C>
__global__ void __launch_bounds__(FF_THREADS) k_ff_partial(const C* p, const unsigned* coords, int nat0, int ndir,
                                                           int nx, int ny, int nz, const float2* tab, int sites_per_block,
                                                           double2* partials) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* st = reinterpret_cast<float2*>(smem_raw);
  const int ntab = nx + ny + nz;
  const int d0 = blockIdx.y * FF_DIRS;
  const int nd = min(FF_DIRS, ndir - d0);
  for (int t = threadIdx.x; t < nd * ntab; t += blockDim.x) st[t] = tab[(size_t)d0 * ntab + t];
  __syncthreads();
  float acc[FF_DIRS][6];
#pragma unroll
  for (int d = 0; d < FF_DIRS; ++d)
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[d][k] = 0.f;
  const int q0 = blockIdx.x * sites_per_block;
  const int q1 = min(nat0, q0 + sites_per_block);
  for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const unsigned pk = coords[q];
    const int ix = pk & 2047u, iy = (pk >> 11) & 2047u, iz = pk >> 22;
    const double2 a = to_d(p[q]), b = to_d(p[q + nat0]), c = to_d(p[q + 2 * (size_t)nat0]);
    const float2 px = make_float2((float)a.x, (float)a.y), py = make_float2((float)b.x, (float)b.y),
                 pz = make_float2((float)c.x, (float)c.y);
#pragma unroll
    for (int d = 0; d < FF_DIRS; ++d) {
      if (d < nd) {
        const float2* td = st + d * ntab;
        const float2 e = cmul(cmul(td[ix], td[nx + iy]), td[nx + ny + iz]);
        const float2 sx = cmul(px, e), sy = cmul(py, e), sz = cmul(pz, e);
        acc[d][0] += sx.x; acc[d][1] += sx.y;
        acc[d][2] += sy.x; acc[d][3] += sy.y;
        acc[d][4] += sz.x; acc[d][5] += sz.y;
      }
    }
  }
  // block reduction in FP64: warp shuffles then shared memory
  __shared__ double red[FF_THREADS / 32][FF_DIRS * 6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < FF_DIRS; ++d)
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double v = (double)acc[d][k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[wid][d * 6 + k] = v;
    }
  __syncthreads();
  for (int t = threadIdx.x; t < nd * 6; t += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < FF_THREADS / 32; ++w) v += red[w][t];
    const int d = t / 6, k = t % 6;
    // partials[(dir)*3 + comp][block] as (re, im)
    double* dst = reinterpret_cast<double*>(&partials[((size_t)(d0 + d) * 3 + k / 2) * gridDim.x + blockIdx.x]);
    dst[k & 1] = v;
  }
}

__global__ void k_ff_final(const double2* partials, int nblocks, int rows, double2* sums) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  double2 s = make_double2(0, 0);
  for (int b = 0; b < nblocks; ++b) {
    const double2 v = partials[(size_t)r * nblocks + b];
    s.x += v.x;
    s.y += v.y;
  }
  sums[r] = s;
}

template <typename T>
int farfield_sums(Engine<T>& eng, const cplx<T>* p, const float* dirs_host, int ndir, const float dx[3], const float x0[3],
                  double2* sums_host, cudaStream_t s) {
  const int nx = eng.g.nx, ny = eng.g.ny, nz = eng.g.nz, nat0 = eng.g.nat0;
  if (nx > 2047 || ny > 2047 || nz > 1023) { set_error("GPU SCAT", "grid too large for packed coordinates"); return 322; }
  const int chunk = 4096;  // directions per launch
  const int sites_per_block = FF_THREADS * 32;
  const int nblocks = (int)ceil_div(nat0, sites_per_block);
  const int ntab = nx + ny + nz;
  unsigned* coords = nullptr;
  double* d_dirs = nullptr;
  float2* tab = nullptr;
  double2 *partials = nullptr, *sums = nullptr;
  int rc = 0;
  cudaError_t e = cudaMalloc((void**)&coords, (size_t)nat0 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_dirs, (size_t)3 * chunk * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&tab, (size_t)chunk * ntab * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&partials, (size_t)chunk * 3 * nblocks * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&sums, (size_t)chunk * 3 * sizeof(double2));
  if (e != cudaSuccess) { set_cuda_error("SCAT workspace", e); rc = 322; }
  if (!rc) {
    k_pack_coords<<<(unsigned)ceil_div(nat0, 256), 256, 0, s>>>(eng.occ, nat0, nx, ny, coords);
    note_launch();
    std::vector<double> hd((size_t)3 * chunk);
    const size_t sm = (size_t)FF_DIRS * ntab * sizeof(float2);
    cudaFuncSetAttribute((const void*)k_ff_partial<cplx<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    for (int off = 0; off < ndir && !rc; off += chunk) {
      const int cnt = std::min(chunk, ndir - off);
      for (int i = 0; i < 3 * cnt; ++i) hd[i] = (double)dirs_host[(size_t)3 * off + i];
      cudaMemcpyAsync(d_dirs, hd.data(), (size_t)3 * cnt * sizeof(double), cudaMemcpyHostToDevice, s);
      k_ff_tables<<<(unsigned)std::min<size_t>(ceil_div((size_t)cnt * ntab, 256), 4096), 256, 0, s>>>(
          d_dirs, cnt, nx, ny, nz, dx[0], dx[1], dx[2], x0[0], x0[1], x0[2], tab);
      note_launch();
      dim3 grid((unsigned)nblocks, (unsigned)ceil_div(cnt, FF_DIRS));
      k_ff_partial<cplx<T>><<<grid, FF_THREADS, sm, s>>>(p, coords, nat0, cnt, nx, ny, nz, tab, sites_per_block, partials);
      note_launch();
      k_ff_final<<<(unsigned)ceil_div((size_t)cnt * 3, 128), 128, 0, s>>>(partials, nblocks, cnt * 3, sums);
      note_launch();
      if (check_launch("SCAT far-field sums")) { rc = 325; break; }
      e = cudaMemcpyAsync(sums_host + (size_t)3 * off, sums, (size_t)3 * cnt * sizeof(double2), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { set_cuda_error("SCAT sums D2H", e); rc = 329; }
    }
  }
  cudaFree(coords); cudaFree(d_dirs); cudaFree(tab); cudaFree(partials); cudaFree(sums);
  return rc;
}

template int evalq_compute<float>(Engine<float>&, VecOps<float>&, const float2*, const float2*, const float2*,
                                  const float2*, int, float2*, double, double2*, double2*);
template int evalq_compute<double>(Engine<double>&, VecOps<double>&, const double2*, const double2*, const double2*,
                                   const double2*, int, double2*, double, double2*, double2*);
template int farfield_sums<float>(Engine<float>&, const float2*, const float*, int, const float[3], const float[3],
                                  double2*, cudaStream_t);
template int farfield_sums<double>(Engine<double>&, const double2*, const float*, int, const float[3], const float[3],
                                   double2*, cudaStream_t);

}  // namespace ddb
