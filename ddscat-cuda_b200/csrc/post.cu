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

// tables[d][0..nx) = exp(-i kx (ix+1+x0x) dx), then ny, then nz entries;
// phases in FP64, stored as complex float (SCAT) or complex double (the
// all-FP64 amplitudes)
template <typename TC>
__global__ void k_ff_tables(const double* dirs, int ndir, int nx, int ny, int nz, double dx0, double dx1, double dx2,
                            double x00, double x01, double x02, TC* tab) {
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
    tab[t] = mk<TC>(c, -s);
  }
}

__global__ void k_pack_coords(const int* occ, int nat0, int nx, int ny, unsigned* packed) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nat0) return;
  const int j = occ[q];
  const unsigned ix = j % nx, iy = (j / nx) % ny, iz = j / (nx * ny);
  packed[q] = ix | (iy << 11) | (iz << 22);
}

// Site position r_j = ((i+1) + x0) * dx of the far-field sums, per axis
struct SitePos {
  float x0[3], dx[3];
};

// Partial sums of ND directions per block: phase products and per-thread
// accumulation in TR (float for SCAT, double for the all-FP64 amplitudes),
// block reduction in FP64.  NS = 3: S_a = sum_j P_ja exp(-i k.r_j); NS = 12
// adds the position moments U_ab = sum_j P_ja r_jb exp(-i k.r_j) (a-major)
// that the scattered angular-momentum flux needs.
template <typename C, typename TR, int ND, int NS = 3>
__global__ void __launch_bounds__(FF_THREADS) k_ff_partial(const C* p, const unsigned* coords, int nat0, int ndir,
                                                           int nx, int ny, int nz, const cplx<TR>* tab,
                                                           int sites_per_block, double2* partials, SitePos pos) {
  using TC = cplx<TR>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TC* st = reinterpret_cast<TC*>(smem_raw);
  const int ntab = nx + ny + nz;
  const int d0 = blockIdx.y * ND;
  const int nd = min(ND, ndir - d0);
  for (int t = threadIdx.x; t < nd * ntab; t += blockDim.x) st[t] = tab[(size_t)d0 * ntab + t];
  __syncthreads();
  constexpr int NA = 2 * NS;  // real accumulators per direction
  TR acc[ND][NA];
#pragma unroll
  for (int d = 0; d < ND; ++d)
#pragma unroll
    for (int k = 0; k < NA; ++k) acc[d][k] = (TR)0;
  const int q0 = blockIdx.x * sites_per_block;
  const int q1 = min(nat0, q0 + sites_per_block);
  for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const unsigned pk = coords[q];
    const int ix = pk & 2047u, iy = (pk >> 11) & 2047u, iz = pk >> 22;
    const double2 a = to_d(p[q]), b = to_d(p[q + nat0]), c = to_d(p[q + 2 * (size_t)nat0]);
    const TC px = mk<TC>(a.x, a.y), py = mk<TC>(b.x, b.y), pz = mk<TC>(c.x, c.y);
    TR rr[3] = {(TR)0, (TR)0, (TR)0};
    if constexpr (NS == 12) {
      rr[0] = ((TR)(ix + 1) + (TR)pos.x0[0]) * (TR)pos.dx[0];
      rr[1] = ((TR)(iy + 1) + (TR)pos.x0[1]) * (TR)pos.dx[1];
      rr[2] = ((TR)(iz + 1) + (TR)pos.x0[2]) * (TR)pos.dx[2];
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      if (d < nd) {
        const TC* td = st + d * ntab;
        const TC e = cmul(cmul(td[ix], td[nx + iy]), td[nx + ny + iz]);
        const TC sa[3] = {cmul(px, e), cmul(py, e), cmul(pz, e)};
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          acc[d][2 * m] += sa[m].x;
          acc[d][2 * m + 1] += sa[m].y;
        }
        if constexpr (NS == 12) {
#pragma unroll
          for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int b2 = 0; b2 < 3; ++b2) {
              acc[d][6 + 6 * m + 2 * b2] += sa[m].x * rr[b2];
              acc[d][7 + 6 * m + 2 * b2] += sa[m].y * rr[b2];
            }
        }
      }
    }
  }
  // block reduction in FP64: warp shuffles then shared memory
  __shared__ double red[FF_THREADS / 32][ND * NA];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d)
#pragma unroll
    for (int k = 0; k < NA; ++k) {
      double v = (double)acc[d][k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) red[wid][d * NA + k] = v;
    }
  __syncthreads();
  for (int t = threadIdx.x; t < nd * NA; t += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < FF_THREADS / 32; ++w) v += red[w][t];
    const int d = t / NA, k = t % NA;
    // partials[(dir)*NS + sum][block] as (re, im)
    double* dst = reinterpret_cast<double*>(&partials[((size_t)(d0 + d) * NS + k / 2) * gridDim.x + blockIdx.x]);
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

// Far-field sums of a compact polarisation p (device) over ndir directions,
// phases and per-thread sums in TR, ND directions per block; NS sums per
// direction (3: S, 12: S and the position moments U), sums_host[dir][NS].
template <typename C, typename TR, int ND, int NS = 3>
static int ff_sums_impl(const int* occ, int nx, int ny, int nz, int nat0, const C* p, const double* dirs_host, int ndir,
                        const double dx[3], const double x0[3], double2* sums_host, cudaStream_t s) {
  using TC = cplx<TR>;
  if (nx > 2047 || ny > 2047 || nz > 1023) { set_error("GPU SCAT", "grid too large for packed coordinates"); return 322; }
  const int chunk = 4096;  // directions per launch
  const int sites_per_block = FF_THREADS * 32;
  const int nblocks = (int)ceil_div(nat0, sites_per_block);
  const int ntab = nx + ny + nz;
  unsigned* coords = nullptr;
  double* d_dirs = nullptr;
  TC* tab = nullptr;
  double2 *partials = nullptr, *sums = nullptr;
  int rc = 0;
  cudaError_t e = cudaMalloc((void**)&coords, (size_t)nat0 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_dirs, (size_t)3 * chunk * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&tab, (size_t)chunk * ntab * sizeof(TC));
  if (e == cudaSuccess) e = cudaMalloc((void**)&partials, (size_t)chunk * NS * nblocks * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&sums, (size_t)chunk * NS * sizeof(double2));
  if (e != cudaSuccess) { set_cuda_error("SCAT workspace", e); rc = 322; }
  if (!rc) {
    k_pack_coords<<<(unsigned)ceil_div(nat0, 256), 256, 0, s>>>(occ, nat0, nx, ny, coords);
    note_launch();
    const size_t sm = (size_t)ND * ntab * sizeof(TC);
    cudaFuncSetAttribute((const void*)k_ff_partial<C, TR, ND, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    SitePos pos;
    for (int k = 0; k < 3; ++k) { pos.x0[k] = (float)x0[k]; pos.dx[k] = (float)dx[k]; }
    for (int off = 0; off < ndir && !rc; off += chunk) {
      const int cnt = std::min(chunk, ndir - off);
      cudaMemcpyAsync(d_dirs, dirs_host + (size_t)3 * off, (size_t)3 * cnt * sizeof(double), cudaMemcpyHostToDevice, s);
      k_ff_tables<TC><<<(unsigned)std::min<size_t>(ceil_div((size_t)cnt * ntab, 256), 4096), 256, 0, s>>>(
          d_dirs, cnt, nx, ny, nz, dx[0], dx[1], dx[2], x0[0], x0[1], x0[2], tab);
      note_launch();
      dim3 grid((unsigned)nblocks, (unsigned)ceil_div(cnt, ND));
      k_ff_partial<C, TR, ND, NS><<<grid, FF_THREADS, sm, s>>>(p, coords, nat0, cnt, nx, ny, nz, tab,
                                                               sites_per_block, partials, pos);
      note_launch();
      k_ff_final<<<(unsigned)ceil_div((size_t)cnt * NS, 128), 128, 0, s>>>(partials, nblocks, cnt * NS, sums);
      note_launch();
      if (check_launch("SCAT far-field sums")) { rc = 325; break; }
      e = cudaMemcpyAsync(sums_host + (size_t)NS * off, sums, (size_t)NS * cnt * sizeof(double2), cudaMemcpyDeviceToHost,
                          s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) { set_cuda_error("SCAT sums D2H", e); rc = 329; }
    }
  }
  cudaFree(coords); cudaFree(d_dirs); cudaFree(tab); cudaFree(partials); cudaFree(sums);
  return rc;
}

template <typename T>
int farfield_sums(Engine<T>& eng, const cplx<T>* p, const float* dirs_host, int ndir, const float dx[3], const float x0[3],
                  double2* sums_host, cudaStream_t s) {
  std::vector<double> hd((size_t)3 * std::max(ndir, 0));
  for (size_t i = 0; i < hd.size(); ++i) hd[i] = (double)dirs_host[i];
  const double dxd[3] = {dx[0], dx[1], dx[2]}, x0d[3] = {x0[0], x0[1], x0[2]};
  return ff_sums_impl<cplx<T>, float, FF_DIRS>(eng.occ, eng.g.nx, eng.g.ny, eng.g.nz, eng.g.nat0, p, hd.data(), ndir,
                                               dxd, x0d, sums_host, s);
}

template <typename T>
int farfield_torque_sums(Engine<T>& eng, const cplx<T>* p, const double* dirs_host, int ndir, const float dx[3],
                         const float x0[3], double2* sums_host, cudaStream_t s) {
  const double dxd[3] = {dx[0], dx[1], dx[2]}, x0d[3] = {x0[0], x0[1], x0[2]};
  return ff_sums_impl<cplx<T>, float, 2, 12>(eng.occ, eng.g.nx, eng.g.ny, eng.g.nz, eng.g.nat0, p, dirs_host, ndir, dxd,
                                             x0d, sums_host, s);
}

// Torque of the incident field E on the dipoles P (compact), per block:
// sum_j 1/2 Re(P_j x conj(E_j)) and sum_j (k/2) Im(P_j . conj(E_j)) r_j x k-hat*|k|,
// six FP64 partials per block, folded in block order by k_torque_final.
template <typename C>
__global__ void __launch_bounds__(256) k_torque_inc(const C* p, const C* e, const int* occ, int nat0, int nx, int ny,
                                                    SitePos pos, double kx, double ky, double kz, double* partials) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nat0; q += gridDim.x * blockDim.x) {
    const int j = occ[q];
    const double r0 = ((j % nx) + 1 + (double)pos.x0[0]) * pos.dx[0];
    const double r1 = (((j / nx) % ny) + 1 + (double)pos.x0[1]) * pos.dx[1];
    const double r2 = ((j / (nx * ny)) + 1 + (double)pos.x0[2]) * pos.dx[2];
    const double2 p0 = to_d(p[q]), p1 = to_d(p[q + nat0]), p2 = to_d(p[q + 2 * (size_t)nat0]);
    const double2 e0 = to_d(e[q]), e1 = to_d(e[q + nat0]), e2 = to_d(e[q + 2 * (size_t)nat0]);
    // Re(a conj(b)) and Im(a conj(b))
    auto rc = [](double2 a, double2 b) { return a.x * b.x + a.y * b.y; };
    auto ic = [](double2 a, double2 b) { return a.y * b.x - a.x * b.y; };
    acc[0] += 0.5 * (rc(p1, e2) - rc(p2, e1));
    acc[1] += 0.5 * (rc(p2, e0) - rc(p0, e2));
    acc[2] += 0.5 * (rc(p0, e1) - rc(p1, e0));
    const double w = 0.5 * (ic(p0, e0) + ic(p1, e1) + ic(p2, e2));
    acc[3] += w * (r1 * kz - r2 * ky);
    acc[4] += w * (r2 * kx - r0 * kz);
    acc[5] += w * (r0 * ky - r1 * kx);
  }
  __shared__ double red[8][6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    partials[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
  }
}

__global__ void k_torque_final(const double* partials, int nblocks, double* out) {
  const int k = threadIdx.x;
  if (k >= 6) return;
  double v = 0.0;
  for (int b = 0; b < nblocks; ++b) v += partials[(size_t)b * 6 + k];
  out[k] = v;
}

// gamma[0..2]: spin part, gamma[3..5]: orbital part of the incident-field torque
template <typename T>
int incident_torque(Engine<T>& eng, const cplx<T>* p, const cplx<T>* e, const float dx[3], const float x0[3],
                    const double k[3], double gamma[6], cudaStream_t s) {
  const int nat0 = eng.g.nat0;
  const int nblocks = (int)std::min<size_t>(ceil_div((size_t)nat0, 256), 1184);
  double* d = nullptr;
  cudaError_t e1 = cudaMalloc((void**)&d, ((size_t)nblocks * 6 + 6) * sizeof(double));
  if (e1 != cudaSuccess) { set_cuda_error("torque workspace", e1); return 341; }
  SitePos pos;
  for (int i = 0; i < 3; ++i) { pos.x0[i] = x0[i]; pos.dx[i] = dx[i]; }
  k_torque_inc<<<(unsigned)nblocks, 256, 0, s>>>(p, e, eng.occ, nat0, eng.g.nx, eng.g.ny, pos, k[0], k[1], k[2], d + 6);
  note_launch();
  k_torque_final<<<1, 32, 0, s>>>(d + 6, nblocks, d);
  note_launch();
  int rc = 0;
  if (check_launch("torque sums")) rc = 342;
  if (!rc) {
    e1 = cudaMemcpyAsync(gamma, d, 6 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(s);
    if (e1 != cudaSuccess) { set_cuda_error("torque sums D2H", e1); rc = 343; }
  }
  cudaFree(d);
  return rc;
}

template int farfield_torque_sums<float>(Engine<float>&, const float2*, const double*, int, const float*, const float*,
                                         double2*, cudaStream_t);
template int incident_torque<float>(Engine<float>&, const float2*, const float2*, const float*, const float*,
                                    const double*, double*, cudaStream_t);

int farfield_sums_f64(const int* occ, int nx, int ny, int nz, int nat0, const double2* p, const double* dirs_host,
                      int ndir, const double dx[3], const double x0[3], double2* sums_host, cudaStream_t s) {
  return ff_sums_impl<double2, double, 4>(occ, nx, ny, nz, nat0, p, dirs_host, ndir, dx, x0, sums_host, s);
}

// --------------------------------------------------------------------------
// Amplitude matrix (S1..S4) and Mueller matrix (S_ij) per scattering direction,
// the step DDSCAT's GETMUELLER performs after SCAT (not in the reference).
// Definitions of Bohren & Huffman (1983), section 3.2 and eq. 3.16; f_ml as
// ddscat_cuda_scat_f32 returns them (k times the physical amplitude), so
// S = -i f.  DDSCAT's basis has EM2 = n x EM1 (phi-hat); Bohren & Huffman's
// perpendicular vector is -EM2 for scattered and incident light, and
// e_par,i = khat x e_perp,i.  With g_1l = f_1l and g_2l = -f_2l:
//   S2 = -i sum_l g_1l conj(e0l).e_par   S3 = -i sum_l g_1l conj(e0l).e_perp
//   S4 = -i sum_l g_2l conj(e0l).e_par   S1 = -i sum_l g_2l conj(e0l).e_perp
struct MuellerIn {
  double kh[3];
  double2 e0c[2][3];  // conj(e01), conj(e02)
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zmulc(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a conj(b)

template <typename R>
__global__ void k_mueller(int ndir, MuellerIn in, const R* em2, const cplx<R>* f11, const cplx<R>* f21,
                          const cplx<R>* f12, const cplx<R>* f22, cplx<R>* s_out, double* m_out) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= ndir) return;
  const double ep[3] = {-(double)em2[3 * d], -(double)em2[3 * d + 1], -(double)em2[3 * d + 2]};  // e_perp = -EM2
  const double ea[3] = {in.kh[1] * ep[2] - in.kh[2] * ep[1], in.kh[2] * ep[0] - in.kh[0] * ep[2],
                        in.kh[0] * ep[1] - in.kh[1] * ep[0]};
  double2 cpar[2], cperp[2];
  for (int l = 0; l < 2; ++l) {
    cpar[l] = make_double2(0.0, 0.0);
    cperp[l] = make_double2(0.0, 0.0);
    for (int k = 0; k < 3; ++k) {
      cpar[l].x += ea[k] * in.e0c[l][k].x; cpar[l].y += ea[k] * in.e0c[l][k].y;
      cperp[l].x += ep[k] * in.e0c[l][k].x; cperp[l].y += ep[k] * in.e0c[l][k].y;
    }
  }
  const double2 a11 = to_d(f11[d]), a12 = to_d(f12[d]);
  const double2 a21 = make_double2(-(double)f21[d].x, -(double)f21[d].y);  // g_2l = -f_2l
  const double2 a22 = make_double2(-(double)f22[d].x, -(double)f22[d].y);
  using C = cplx<R>;
  auto mi = [](double2 z) { return make_double2(z.y, -z.x); };  // -i z
  auto add = [](double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); };
  const double2 S2 = mi(add(zmul(a11, cpar[0]), zmul(a12, cpar[1])));
  const double2 S3 = mi(add(zmul(a11, cperp[0]), zmul(a12, cperp[1])));
  const double2 S4 = mi(add(zmul(a21, cpar[0]), zmul(a22, cpar[1])));
  const double2 S1 = mi(add(zmul(a21, cperp[0]), zmul(a22, cperp[1])));
  if (s_out) {
    s_out[4 * d] = mk<C>(S1.x, S1.y);
    s_out[4 * d + 1] = mk<C>(S2.x, S2.y);
    s_out[4 * d + 2] = mk<C>(S3.x, S3.y);
    s_out[4 * d + 3] = mk<C>(S4.x, S4.y);
  }
  const double q1 = zabs2(S1), q2 = zabs2(S2), q3 = zabs2(S3), q4 = zabs2(S4);
  const double2 s23 = zmulc(S2, S3), s14 = zmulc(S1, S4), s24 = zmulc(S2, S4), s13 = zmulc(S1, S3);
  const double2 s12 = zmulc(S1, S2), s34 = zmulc(S3, S4);
  double* M = m_out + (size_t)16 * d;
  M[0] = 0.5 * (q2 + q1 + q4 + q3);
  M[1] = 0.5 * (q2 - q1 + q4 - q3);
  M[2] = s23.x + s14.x;
  M[3] = s23.y - s14.y;
  M[4] = 0.5 * (q2 - q1 - q4 + q3);
  M[5] = 0.5 * (q2 + q1 - q4 - q3);
  M[6] = s23.x - s14.x;
  M[7] = s23.y + s14.y;
  M[8] = s24.x + s13.x;
  M[9] = s24.x - s13.x;
  M[10] = s12.x + s34.x;
  M[11] = -s12.y - s34.y;   // Im(S2 S1* + S4 S3*)
  M[12] = -s24.y + s13.y;   // Im(S4 S2* + S1 S3*)
  M[13] = -s24.y - s13.y;   // Im(S4 S2* - S1 S3*)
  M[14] = s12.y - s34.y;    // Im(S1 S2* - S3 S4*)
  M[15] = s12.x - s34.x;
}

template <typename R>
static int mueller_impl(int ndir, const R* ak, const cplx<R>* e01, const cplx<R>* e02, const R* em2, const cplx<R>* f11,
                        const cplx<R>* f21, const cplx<R>* f12, const cplx<R>* f22, cplx<R>* s_out, double* m_out) {
  using C = cplx<R>;
  MuellerIn in{};
  const double kk = std::sqrt((double)ak[0] * ak[0] + (double)ak[1] * ak[1] + (double)ak[2] * ak[2]);
  if (!(kk > 0.0)) { set_error("Mueller", "zero incident wave vector"); return 700; }
  for (int k = 0; k < 3; ++k) {
    in.kh[k] = ak[k] / kk;
    in.e0c[0][k] = make_double2(e01[k].x, -e01[k].y);
    in.e0c[1][k] = make_double2(e02[k].x, -e02[k].y);
  }
  const size_t off_f = ((size_t)ndir * 3 * sizeof(R) + 15) & ~(size_t)15;  // 16-byte aligned f block
  const size_t nb = off_f + (size_t)ndir * (8 * sizeof(C) + 16 * sizeof(double));
  unsigned char* buf = nullptr;
  cudaError_t e = cudaMalloc((void**)&buf, nb);
  if (e != cudaSuccess) { set_cuda_error("Mueller workspace", e); return 701; }
  R* d_em2 = reinterpret_cast<R*>(buf);
  C* d_f = reinterpret_cast<C*>(buf + off_f);
  C* d_s = d_f + (size_t)4 * ndir;
  double* d_m = reinterpret_cast<double*>(d_s + (size_t)4 * ndir);
  const C* hf[4] = {f11, f21, f12, f22};
  e = cudaMemcpy(d_em2, em2, (size_t)ndir * 3 * sizeof(R), cudaMemcpyHostToDevice);
  for (int k = 0; k < 4 && e == cudaSuccess; ++k)
    e = cudaMemcpy(d_f + (size_t)k * ndir, hf[k], (size_t)ndir * sizeof(C), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { cudaFree(buf); set_cuda_error("Mueller H2D", e); return 702; }
  k_mueller<R><<<(unsigned)ceil_div(ndir, 128), 128>>>(ndir, in, d_em2, d_f, d_f + ndir, d_f + 2 * (size_t)ndir,
                                                       d_f + 3 * (size_t)ndir, d_s, d_m);
  note_launch();
  if (check_launch("Mueller kernel")) { cudaFree(buf); return 703; }
  if (s_out) e = cudaMemcpy(s_out, d_s, (size_t)ndir * 4 * sizeof(C), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(m_out, d_m, (size_t)ndir * 16 * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) { set_cuda_error("Mueller D2H", e); return 702; }
  return 0;
}

int mueller_compute(int ndir, const float* ak, const float2* e01, const float2* e02, const float* em2,
                    const float2* f11, const float2* f21, const float2* f12, const float2* f22, float2* s_out,
                    double* m_out) {
  return mueller_impl<float>(ndir, ak, e01, e02, em2, f11, f21, f12, f22, s_out, m_out);
}

int mueller_compute_f64(int ndir, const double* ak, const double2* e01, const double2* e02, const double* em2,
                        const double2* f11, const double2* f21, const double2* f12, const double2* f22,
                        double2* s_out, double* m_out) {
  return mueller_impl<double>(ndir, ak, e01, e02, em2, f11, f21, f12, f22, s_out, m_out);
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
