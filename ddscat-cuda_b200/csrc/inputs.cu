// Right-hand sides and diagonal blocks generated on the GPU (library
// extension, no counterpart in the reference: DDSCAT computes them on the host
// in EVALE and ALPHADIAG and passes them to the solver entry points).
//
// For right-hand side r with wave vector k_r (lattice units, d = 1) and
// polarisation e_r, and each lattice site j = ix + nx*(iy + ny*iz):
//   b[r][c][j]    = e_r[c] exp(i k_r . r_j) on occupied sites, 0 on vacuum,
//                   r_j = (ix+1, iy+1, iz+1) + x0 (the SCAT convention, cu:805)
//   adia[r][c][j] = 1/alpha_c(m of the site's material, |k_r|, khat_r, e_r)
// with one of DDSCAT's polarisability prescriptions (CMDPOL), lattice units
// d = 1, 1/alpha_CM = (4pi/3)(m^2+2)/(m^2-1):
//   LATTDR (Draine & Goodman 1993, ApJ 405, 685): 1/alpha = 1/alpha_CM +
//     (b1 + m^2 b2 + m^2 b3 S)(kd)^2 - (2/3) i (kd)^3, S = sum_a (khat_a Re e_a)^2,
//     b1 = -1.891531, b2 = 0.1648469, b3 = -1.7700004, the same for c = 1..3;
//   GKDLDR (Gutkowicz-Krusin & Draine 2004): the same with S replaced by
//     khat_c^2 for component c (independent of the polarisation);
//   FLTRCD (filtered coupled dipoles; Piller & Martin 1998, Gay-Balmaz &
//     Martin 2002): 1/alpha = 1/alpha_CM - (4/3)(kd)^2
//     - (2/(3 pi)) ln((pi - kd)/(pi + kd)) (kd)^3 - (2/3) i (kd)^3, kd < pi.
// The 1/alpha table (nrhs x materials x 3 components) is computed in FP64 on
// the host; the phases are evaluated in FP64 on the GPU.
#include <cmath>
#include <complex>
#include <vector>
#include "ddscat_b200.h"
#include "engine.h"

namespace ddb {

__global__ void k_make_inputs(int nx, int ny, int nat, int nrhs, const double* kv, const double2* e0, double x00,
                              double x01, double x02, const int16_t* iocc, const int16_t* icomp, int nmat1,
                              const float2* adtab, float2* b, float2* adia) {
  const int r = blockIdx.y;
  const double kx = kv[3 * r], ky = kv[3 * r + 1], kz = kv[3 * r + 2];
  const double2 ex = e0[3 * r], ey = e0[3 * r + 1], ez = e0[3 * r + 2];
  float2* br = b ? b + (size_t)r * 3 * nat : nullptr;
  float2* ar = adia ? adia + (size_t)r * 3 * nat : nullptr;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nat; j += gridDim.x * blockDim.x) {
    const int ix = j % nx, iy = (j / nx) % ny, iz = j / (nx * ny);
    const bool occ = iocc[j] != 0;
    if (br) {
      float2 v0 = make_float2(0.f, 0.f), v1 = v0, v2 = v0;
      if (occ) {
        const double ph = kx * (ix + 1 + x00) + ky * (iy + 1 + x01) + kz * (iz + 1 + x02);
        double sn, cs;
        sincos(ph, &sn, &cs);
        v0 = make_float2((float)(ex.x * cs - ex.y * sn), (float)(ex.x * sn + ex.y * cs));
        v1 = make_float2((float)(ey.x * cs - ey.y * sn), (float)(ey.x * sn + ey.y * cs));
        v2 = make_float2((float)(ez.x * cs - ez.y * sn), (float)(ez.x * sn + ez.y * cs));
      }
      br[j] = v0;
      br[(size_t)nat + j] = v1;
      br[2 * (size_t)nat + j] = v2;
    }
    if (ar) {
      const int mat = (occ && icomp) ? icomp[j] : 1;
      const float2* a = adtab + ((size_t)r * nmat1 + mat) * 3;
      ar[j] = a[0];
      ar[(size_t)nat + j] = a[1];
      ar[2 * (size_t)nat + j] = a[2];
    }
  }
}

// host: 1/alpha per Cartesian component c for one (rhs, material); material 0
// is unused (vacuum).  Returns false for FLTRCD with kd >= pi.
static bool inv_alpha(int cmdpol, std::complex<double> m, double kd, const double* khat,
                      const std::complex<double>* e, std::complex<double> out[3]) {
  const double b1 = -1.891531, b2 = 0.1648469, b3 = -1.7700004;
  const double pi = 3.14159265358979323846;
  const std::complex<double> eps = m * m;
  const std::complex<double> base =
      (4.0 * pi / 3.0) * (eps + 2.0) / (eps - 1.0) - std::complex<double>(0.0, 2.0 / 3.0) * kd * kd * kd;
  if (cmdpol == DDSCAT_B200_FLTRCD) {
    if (!(kd < pi)) return false;
    const double corr = -(4.0 / 3.0) * kd * kd - (2.0 / (3.0 * pi)) * std::log((pi - kd) / (pi + kd)) * kd * kd * kd;
    for (int c = 0; c < 3; ++c) out[c] = base + corr;
    return true;
  }
  double S = 0.0;
  for (int a = 0; a < 3; ++a) S += (khat[a] * e[a].real()) * (khat[a] * e[a].real());
  for (int c = 0; c < 3; ++c) {
    const double Sc = cmdpol == DDSCAT_B200_GKDLDR ? khat[c] * khat[c] : S;
    out[c] = base + (b1 + eps * b2 + eps * b3 * Sc) * kd * kd;
  }
  return true;
}

int make_inputs(const Engine<float>& eng, int cmdpol, int nrhs, const float* k, const float2* e0, const float* x0,
                int nmat, const float2* mref, const int16_t* icomp_host, float2* b, float2* adia, cudaStream_t st) {
  const Geometry& g = eng.g;
  if (cmdpol != DDSCAT_B200_LATTDR && cmdpol != DDSCAT_B200_GKDLDR && cmdpol != DDSCAT_B200_FLTRCD) {
    set_error("make_inputs", "unknown polarisability prescription (LATTDR=0, GKDLDR=1, FLTRCD=2)");
    return 610;
  }
  std::vector<double> kv((size_t)3 * nrhs);
  std::vector<double2> ev((size_t)3 * nrhs);
  std::vector<float2> tab((size_t)nrhs * (nmat + 1) * 3, make_float2(0.f, 0.f));
  for (int r = 0; r < nrhs; ++r) {
    double kh[3], kk = 0.0;
    std::complex<double> e[3];
    for (int a = 0; a < 3; ++a) {
      kv[3 * r + a] = k[3 * r + a];
      kk += kv[3 * r + a] * kv[3 * r + a];
      e[a] = std::complex<double>(e0[3 * r + a].x, e0[3 * r + a].y);
      ev[3 * r + a] = make_double2(e[a].real(), e[a].imag());
    }
    kk = std::sqrt(kk);
    if (!(kk > 0.0)) { set_error("make_inputs", "zero wave vector"); return 610; }
    for (int a = 0; a < 3; ++a) kh[a] = kv[3 * r + a] / kk;
    for (int mi = 1; mi <= nmat; ++mi) {
      std::complex<double> ia[3];
      if (!inv_alpha(cmdpol, std::complex<double>(mref[mi - 1].x, mref[mi - 1].y), kk, kh, e, ia)) {
        set_error("make_inputs", "FLTRCD needs |k| d < pi");
        return 610;
      }
      for (int c = 0; c < 3; ++c)
        tab[((size_t)r * (nmat + 1) + mi) * 3 + c] = make_float2((float)ia[c].real(), (float)ia[c].imag());
    }
  }
  if (icomp_host) {
    for (int j = 0; j < g.nat; ++j)
      if (icomp_host[j] < 0 || icomp_host[j] > nmat) {
        set_error("make_inputs", "material index outside 1..nmat (or 0 for vacuum)");
        return 611;
      }
  }
  double* d_k = nullptr;
  double2* d_e = nullptr;
  float2* d_tab = nullptr;
  int16_t* d_icomp = nullptr;
  cudaError_t e = cudaMalloc((void**)&d_k, kv.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_e, ev.size() * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_tab, tab.size() * sizeof(float2));
  if (e == cudaSuccess && icomp_host) e = cudaMalloc((void**)&d_icomp, (size_t)g.nat * sizeof(int16_t));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_k, kv.data(), kv.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_e, ev.data(), ev.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(float2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && icomp_host)
    e = cudaMemcpyAsync(d_icomp, icomp_host, (size_t)g.nat * sizeof(int16_t), cudaMemcpyHostToDevice, st);
  int rc = 0;
  if (e != cudaSuccess) {
    set_cuda_error("make_inputs buffers", e);
    rc = 612;
  } else {
    const unsigned gx = (unsigned)std::min<size_t>(ceil_div((size_t)g.nat, 256), std::max(1, 1184 / nrhs));
    k_make_inputs<<<dim3(gx, (unsigned)nrhs), 256, 0, st>>>(g.nx, g.ny, g.nat, nrhs, d_k, d_e, x0[0], x0[1], x0[2],
                                                            eng.iocc, d_icomp, nmat + 1, d_tab, b, adia);
    note_launch();
    if (check_launch("make_inputs")) rc = 613;
    else if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { set_cuda_error("make_inputs", e); rc = 613; }
  }
  cudaFree(d_k); cudaFree(d_e); cudaFree(d_tab); cudaFree(d_icomp);
  return rc;
}

}  // namespace ddb
