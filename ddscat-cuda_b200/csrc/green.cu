// On-GPU construction of the FFT'd Green tensor (sm_100a).
//
// Follows ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu:600-652: the direct
// interaction at every lag of the 2n padded grid (point dipole IDIPINT=0 or
// filtered coupled dipole IDIPINT=1, periodic replica sums for IPBC=1, lag n
// set to zero), transformed with exp(+i) and, for IPBC=0, trimmed to the
// (n+1)^3 octant.  Here the lag values are generated inside the x-axis FFT
// kernel (no M^3 scratch for the direct sum), all three transforms run in FP64
// and the result is rounded once to the engine precision; the y and z
// transforms produce only the n+1 outputs the octant keeps.
#include <algorithm>
#include "engine.h"

namespace ddb {

struct GreenDev {
  int nx, ny, nz, Mx, My, Mz, ipbc, idipint;
  double gamma, akx, aky, akz, dx1, dx2, dx3, akd, akd2, pyddx, pzddx;
};

// Cosine and sine integrals Ci(t), Si(t) for t >= 0: power series for t <= 2,
// otherwise the continued fraction of E1(i t) = -Ci(t) + i (Si(t) - pi/2)
// evaluated with the modified Lentz method (Press et al., Numerical Recipes,
// section 6.9).  Returns false if the iteration does not converge.
__device__ bool ci_si(double t, double& ci, double& si) {
  const double euler = 0.57721566490153286061, half_pi = 1.57079632679489661923;
  if (t <= 0.0) { ci = -1.0e300; si = 0.0; return true; }
  if (t <= 2.0) {
    // Si = sum (-1)^k t^(2k+1) / ((2k+1) (2k+1)!),  Ci = gamma + ln t + sum_{k>=1} (-1)^k t^(2k) / (2k (2k)!)
    double s = 0.0, c = 0.0, term = t;  // term = t^(m) / m!
    bool ok = false;
    for (int m = 1; m <= 200; ++m) {
      // term holds t^m / m!
      double add;
      if (m & 1) {
        const int k = (m - 1) / 2;
        add = ((k & 1) ? -1.0 : 1.0) * term / m;
        s += add;
      } else {
        const int k = m / 2;
        add = ((k & 1) ? -1.0 : 1.0) * term / m;
        c += add;
      }
      if (fabs(add) < 1e-17 * (fabs(s) + fabs(c) + 1e-300) && m > 2) { ok = true; break; }
      term *= t / (m + 1);
    }
    si = s;
    ci = euler + log(t) + c;
    return ok;
  }
  // modified Lentz on b0 = 1 + i t, a_k = -k^2, b_k = b_{k-1} + 2
  const double tiny = 1e-300;
  double br = 1.0, bi = t;
  double cr = 1.0 / tiny, ci_ = 0.0;
  double den = br * br + bi * bi;
  double dr = br / den, di = -bi / den;  // d = 1/b
  double hr = dr, hi = di;
  bool ok = false;
  for (int k = 1; k <= 500; ++k) {
    const double a = -(double)k * (double)k;
    br += 2.0;
    // d = 1 / (a d + b)
    double xr = a * dr + br, xi = a * di + bi;
    den = xr * xr + xi * xi;
    dr = xr / den; di = -xi / den;
    // c = b + a / c
    den = cr * cr + ci_ * ci_;
    double qr = a * cr / den, qi = -a * ci_ / den;
    cr = br + qr; ci_ = bi + qi;
    // h *= c d
    const double er = cr * dr - ci_ * di, ei = cr * di + ci_ * dr;
    const double nhr = hr * er - hi * ei, nhi = hr * ei + hi * er;
    hr = nhr; hi = nhi;
    if (fabs(er - 1.0) + fabs(ei) < 1e-16) { ok = true; break; }
  }
  // E1(it) = e^{-it} h
  const double cs = cos(t), sn = sin(t);
  const double er = cs * hr + sn * hi, ei = cs * hi - sn * hr;
  ci = -er;
  si = half_pi + ei;
  return ok;
}

// Accumulate the six components (xx,xy,xz,yy,yz,zz) of the interaction at
// separation (x,y,z); cu:622-633.
__device__ void green_interaction(double x, double y, double z, double phasyz, double damp, const GreenDev& p, double2 c[6],
                                  int* status) {
  const double r2 = x * x + y * y + z * z;
  if (r2 <= 1.0e-6) return;
  const double r = sqrt(r2), r3 = r * r2, kr = p.akd * r;
  const double xx[3] = {x, y, z};
  if (p.idipint == 0) {
    double sn, cs;
    sincos(kr + phasyz, &sn, &cs);
    const double e = exp(-damp) / r3;
    const double2 ph = make_double2(e * cs, e * sn);
    const double2 fac = make_double2(1.0 / r2, -kr / r2);  // (1 - i kr) / r^2
    int m = 0;
    for (int ii = 0; ii < 3; ++ii) {
      const double q = xx[ii] * xx[ii];
      const double2 term = make_double2(p.akd2 * (q - r2) + fac.x * (r2 - 3.0 * q), fac.y * (r2 - 3.0 * q));
      c[m] = csub(c[m], cmul(ph, term));
      ++m;
      for (int jj = ii + 1; jj < 3; ++jj) {
        const double2 t2 = make_double2(p.akd2 - 3.0 * fac.x, -3.0 * fac.y);
        c[m] = csub(c[m], cscale(cmul(ph, t2), xx[ii] * xx[jj]));
        ++m;
      }
    }
  } else if (p.idipint == 1) {
    const double pi = 3.14159265358979323846, kfr = pi * r;
    double cip, sip, cim, sim;
    const double am = kfr - kr;
    if (!ci_si(kfr + kr, cip, sip) || !ci_si(fabs(am), cim, sim)) { atomicCAS(status, 0, 11); return; }
    if (am < 0.0) sim = -sim;
    double sinkr, coskr, sinkfr, coskfr;
    sincos(kr, &sinkr, &coskr);
    sincos(kfr, &sinkfr, &coskfr);
    const double a0 = sinkr * (cip - cim) + coskr * (pi - sip - sim);
    const double a1 = p.akd * sinkr * (-pi + sip + sim) + p.akd * coskr * (cip - cim) - 2.0 * sinkfr / r;
    const double a2 = p.akd2 * (sinkr * (cim - cip) + coskr * (sip + sim - pi)) + 2.0 * (sinkfr - kfr * coskfr) / r2;
    const double2 eikr = make_double2(coskr, sinkr);
    double sp, cp;
    sincos(phasyz, &sp, &cp);
    const double ed = exp(-damp);
    const double2 ph = make_double2(ed * cp, ed * sp);
    const double2 g0 = cscale(make_double2(eikr.x - a0 / pi, eikr.y), 1.0 / r);
    const double2 g1 = cscale(cadd(cmul(eikr, make_double2(-1.0, kr)), make_double2((a0 - a1 * r) / pi, 0.0)), 1.0 / r2);
    const double2 g2 = cscale(csub(cmul(eikr, make_double2(2.0 - kr * kr, -2.0 * kr)),
                                   make_double2((2.0 * (a0 - r * a1) + r2 * a2) / pi, 0.0)),
                              1.0 / r3);
    const double h2 = (sinkfr - kfr * coskfr) / (pi * r3);
    const double2 radial = csub(cscale(g2, 1.0 / r2), cscale(g1, 1.0 / r3));
    int m = 0;
    for (int ii = 0; ii < 3; ++ii) {
      double2 base = cadd(cadd(cscale(g0, p.akd2), cscale(g1, 1.0 / r)), make_double2((2.0 / 3.0) * h2, 0.0));
      base = cadd(base, cscale(radial, xx[ii] * xx[ii]));
      c[m] = cadd(c[m], cmul(ph, base));
      ++m;
      for (int jj = ii + 1; jj < 3; ++jj) {
        c[m] = cadd(c[m], cscale(cmul(ph, radial), xx[ii] * xx[jj]));
        ++m;
      }
    }
  } else {
    atomicCAS(status, 0, 12);
  }
}

// Direct Green sum at integer lag (lx,ly,lz), including the periodic replica
// sums with the Gaussian-type damping of cu:634-643.
__device__ void green_sum_lag(int lx, int ly, int lz, const GreenDev& p, double2 c[6], int* status) {
  for (int m = 0; m < 6; ++m) c[m] = make_double2(0.0, 0.0);
  const double x0 = lx * p.dx1, y0 = ly * p.dx2, z0 = lz * p.dx3;
  int jpbc = 0, jpy1 = 0, jpy2 = 0, jpz1 = 0, jpz2 = 0;
  double kperp = 0, krf = 0, phasf = 0;
  if (p.ipbc > 0) {
    double kp2;
    if (p.pyddx <= 0.0) { jpbc = 2; kp2 = p.akx * p.akx + p.aky * p.aky; }
    else if (p.pzddx <= 0.0) { jpbc = 1; kp2 = p.akx * p.akx + p.akz * p.akz; }
    else { jpbc = 3; kp2 = p.akx * p.akx; }
    if (kp2 <= 0.0) { atomicCAS(status, 0, 13); return; }
    kperp = sqrt(kp2);
    const double phimax = 1.0 / p.gamma;
    const double term0 = p.akd2 * phimax * phimax / kp2, term1 = 2.0 * p.akd * phimax;
    const double term2y = p.aky * phimax / kp2, term2z = p.akz * phimax / kp2;
    if (jpbc == 1) {
      const double rperp = sqrt(x0 * x0 + z0 * z0);
      krf = p.akd2 * rperp / kperp;
      const double yf = y0 - p.aky * rperp / kperp;
      phasf = p.aky * yf;
      const double term3 = sqrt(term0 + term1 * rperp) / kperp;
      jpy1 = (int)((yf - term2y - term3) / p.pyddx + 0.999999);
      jpy2 = (int)((yf - term2y + term3) / p.pyddx);
    } else if (jpbc == 2) {
      const double rperp = sqrt(x0 * x0 + y0 * y0);
      krf = p.akd2 * rperp / kperp;
      const double zf = z0 - p.akz * rperp / kperp;
      phasf = p.akz * zf;
      const double term3 = sqrt(term0 + term1 * rperp) / kperp;
      jpz1 = (int)((zf - term2z - term3) / p.pzddx + 0.999999);
      jpz2 = (int)((zf - term2z + term3) / p.pzddx);
    } else {
      const double rperp = fabs(x0);
      krf = p.akd2 * rperp / kperp;
      const double yf = y0 - p.aky * rperp / kperp, zf = z0 - p.akz * rperp / kperp;
      phasf = p.aky * yf + p.akz * zf;
      const double term3 = sqrt(term0 + term1 * rperp) / kperp;
      jpy1 = (int)((yf - term2y - term3) / p.pyddx + 0.999999);
      jpy2 = (int)((yf - term2y + term3) / p.pyddx);
      jpz1 = (int)((zf - term2z - term3) / p.pzddx + 0.999999);
      jpz2 = (int)((zf - term2z + term3) / p.pzddx);
    }
  }
  const double phimax = (p.gamma > 0.0) ? 1.0 / p.gamma : 0.0;
  const double beta = (p.ipbc > 0) ? 16.0 / (phimax * phimax * phimax * phimax) : 0.0;
  for (int jpy = jpy1; jpy <= jpy2; ++jpy) {
    const double rjpy = jpy * p.pyddx * p.dx2, y = y0 - rjpy, phasy = p.aky * rjpy;
    for (int jpz = jpz1; jpz <= jpz2; ++jpz) {
      const double rjpz = jpz * p.pzddx * p.dx3, z = z0 - rjpz;
      const double r2 = x0 * x0 + y * y + z * z;
      if (r2 <= 1.0e-6) continue;
      const double kr = p.akd * sqrt(r2), phasyz = phasy + p.akz * rjpz;
      double damp = 0.0;
      if (jpbc != 0) {
        const double phi = kr - krf + phasyz - phasf;
        damp = beta * phi * phi * phi * phi;
      }
      green_interaction(x0, y, z, phasyz, damp, p, c, status);
    }
  }
}

// x pass: one lag row (iy, iz) for all 6 components, FFT(+i) along x in FP64,
// keep the first nxo outputs.  out[m][iz][iy][kx], dims (6, Mz, My, nxo).
__global__ void __launch_bounds__(256) k_green_x(GreenDev p, FftPlan plan, const double2* tw, double2* out, int nxo,
                                                 int* status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int Mx = p.Mx, My = p.My, Mz = p.Mz, LD = Mx + 1;
  double2* A = reinterpret_cast<double2*>(smem_raw);
  double2* B = A + 6 * LD;
  const int iy = blockIdx.x, iz = blockIdx.y;
  for (int ix = threadIdx.x; ix < Mx; ix += blockDim.x) {
    double2 c[6];
    // lags -(n-1)..n-1 at FFT indices 0..n-1 and M-n+1..M-1; the indices
    // between (lag n for M = 2n, cu:644) are zero
    const bool gap = (ix >= p.nx && ix <= Mx - p.nx) || (iy >= p.ny && iy <= My - p.ny) ||
                     (iz >= p.nz && iz <= Mz - p.nz);
    if (gap) {
      for (int m = 0; m < 6; ++m) c[m] = make_double2(0.0, 0.0);
    } else {
      const int lx = ix < p.nx ? ix : ix - Mx, ly = iy < p.ny ? iy : iy - My, lz = iz < p.nz ? iz : iz - Mz;
      green_sum_lag(lx, ly, lz, p, c, status);
    }
    for (int m = 0; m < 6; ++m) A[m * LD + ix] = c[m];
  }
  __syncthreads();
  double2* R = fft_tile<+1>(A, B, Lay{LD, 1}, 6, plan, tw);
  for (int t = threadIdx.x; t < 6 * nxo; t += blockDim.x) {
    const int m = t / nxo, kx = t % nxo;
    out[(((size_t)m * Mz + iz) * My + iy) * nxo + kx] = R[m * LD + kx];
  }
}

// Column FFT: in[b][e][w] (e < L rows, W columns) -> FFT(+i) along e ->
// out[b][e][w] for e < Lout.  Used for the y and z transforms of the Green tensor.
template <typename Tout>
__global__ void __launch_bounds__(256) k_green_col(const double2* in, Tout* out, int L, int W, int Lout, FftPlan plan,
                                                   const double2* tw, int TX) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2* A = reinterpret_cast<double2*>(smem_raw);
  double2* B = A + (size_t)TX * L;
  const int w0 = blockIdx.x * TX;
  const size_t b = blockIdx.y;
  const double2* src = in + b * (size_t)L * W;
  for (int t = threadIdx.x; t < TX * L; t += blockDim.x) {
    const int l = t % TX, e = t / TX, w = w0 + l;
    A[e * TX + l] = (w < W) ? src[(size_t)e * W + w] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  double2* R = fft_tile<+1>(A, B, Lay{1, TX}, TX, plan, tw);
  Tout* dst = out + b * (size_t)Lout * W;
  for (int t = threadIdx.x; t < TX * Lout; t += blockDim.x) {
    const int l = t % TX, e = t / TX, w = w0 + l;
    if (w < W) dst[(size_t)e * W + w] = from_d<Tout>(R[e * TX + l]);
  }
}

static double2* twiddles_d(int n) {
  std::vector<double2> h(n);
  const double pi = 3.14159265358979323846;
  for (int m = 0; m < n; ++m) h[m] = make_double2(std::cos(-2.0 * pi * m / n), std::sin(-2.0 * pi * m / n));
  double2* d = nullptr;
  if (cudaMalloc((void**)&d, n * sizeof(double2)) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
  return d;
}

template <typename T> int Engine<T>::build_green(const GreenArgs<T>& ga) {
  GreenDev p{};
  p.nx = g.nx; p.ny = g.ny; p.nz = g.nz; p.Mx = g.Mx; p.My = g.My; p.Mz = g.Mz;
  p.ipbc = g.ipbc; p.idipint = ga.idipint;
  p.gamma = ga.gamma;
  p.akx = ga.ak[0]; p.aky = ga.ak[1]; p.akz = ga.ak[2];
  p.dx1 = ga.dx[0]; p.dx2 = ga.dx[1]; p.dx3 = ga.dx[2];
  p.akd = std::sqrt(p.akx * p.akx + p.aky * p.aky + p.akz * p.akz);
  p.akd2 = p.akd * p.akd;
  p.pyddx = ga.pyd * ga.dx[1];
  p.pzddx = ga.pzd * ga.dx[2];
  const int Mx = g.Mx, My = g.My, Mz = g.Mz;
  const int nxo = g.ipbc == 0 ? Mx / 2 + 1 : Mx, nyo = g.ipbc == 0 ? My / 2 + 1 : My, nzo = g.ipbc == 0 ? Mz / 2 + 1 : Mz;
  double2 *twx_d = twiddles_d(Mx), *twy_d = twiddles_d(My), *twz_d = twiddles_d(Mz);
  double2 *a1 = nullptr, *a2 = nullptr;
  int* d_status = nullptr;
  int rc = 0;
  cudaError_t e = cudaMalloc((void**)&a1, (size_t)6 * Mz * My * nxo * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&a2, (size_t)6 * Mz * nyo * nxo * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_status, sizeof(int));
  if (e != cudaSuccess || !twx_d || !twy_d || !twz_d) {
    set_cuda_error("Green temporary allocation", e);
    rc = 2;
  } else {
    cudaMemset(d_status, 0, sizeof(int));
    const size_t smx = (size_t)2 * 6 * (Mx + 1) * sizeof(double2);
    cudaFuncSetAttribute((const void*)k_green_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    k_green_x<<<dim3(My, Mz), 256, smx>>>(p, px, twx_d, a1, nxo, d_status);
    note_launch();
    if (check_launch("Green direct sum + x FFT")) rc = 4;
    const FftPlan ply = make_fft_plan(My), plz = make_fft_plan(Mz);
    if (!rc) {
      const int TX = std::max(1, std::min(32, 4096 / My));
      const size_t sm = (size_t)2 * TX * My * sizeof(double2);
      cudaFuncSetAttribute((const void*)k_green_col<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      k_green_col<double2><<<dim3((unsigned)ceil_div(nxo, TX), 6 * Mz), 256, sm>>>(a1, a2, My, nxo, nyo, ply, twy_d, TX);
      note_launch();
      if (check_launch("Green y FFT")) rc = 5;
    }
    if (!rc) {
      const int W = nyo * nxo;
      const int TX = std::max(1, std::min(32, 4096 / Mz));
      const size_t sm = (size_t)2 * TX * Mz * sizeof(double2);
      cudaFuncSetAttribute((const void*)k_green_col<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      C* planar = reinterpret_cast<C*>(a1);  // a1 is free now and larger than the result
      k_green_col<C><<<dim3((unsigned)ceil_div(W, TX), 6), 256, sm>>>(a2, planar, Mz, W, nzo, plz, twz_d, TX);
      note_launch();
      if (check_launch("Green z FFT")) rc = 6;
      if (!rc && interleave_green(planar)) rc = 6;
    }
    e = cudaDeviceSynchronize();
    if (!rc && e != cudaSuccess) { set_cuda_error("Green build synchronize", e); rc = 7; }
    int h_status = 0;
    if (!rc) cudaMemcpy(&h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (!rc && h_status) {
      char msg[160];
      std::snprintf(msg, sizeof(msg), "Green kernel status=%d (11=CISI,12=IDIPINT,13=KPERP)", h_status);
      set_error("CUDA Green", msg);
      rc = 14;
    }
  }
  cudaFree(a1); cudaFree(a2); cudaFree(d_status);
  cudaFree(twx_d); cudaFree(twy_d); cudaFree(twz_d);
  return rc;
}

template int Engine<float>::build_green(const GreenArgs<float>&);
template int Engine<double>::build_green(const GreenArgs<double>&);

}  // namespace ddb
