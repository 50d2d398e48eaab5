"""CPU oracle for the DDSCAT DDA solve path -- TEST INFRASTRUCTURE ONLY.

This module is the checker.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import it.  The product path
(``ddscat-cuda_b200``) never calls into it and fails loudly when its CUDA
library is missing.

It restates, in NumPy (FP64 unless a function says otherwise), the algorithm of
the reference CUDA backend ``ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu``
(cited below as ``cu:<line>``) and the CPU operator specification in
``ddscat_cuda_unified/fortran/cprod_cuda.f90`` (``cprod:<line>``).  Every
function names the lines it follows.

Parity pinning: the reference publishes no golden vectors for results.  Its two
numeric scripts (``scripts/check_compact_mapping.py`` and
``scripts/test_gpu_final_sections_math.py``) are restated as tests, and the
reference library itself, compiled from its unmodified sources by
``oracle/Makefile`` into ``oracle/_ref/``, is run on a B200 by
``tests/golden/make_reference_fixtures.py``; the committed fixtures under
``tests/golden/`` pin this oracle (``tests/test_oracle_pinned.py``).

Layout conventions (the reference's, ``cu:107``, ``cu:122``):
  full vector  v[j + m*NAT], j = ix + nx*(iy + ny*iz), m = 0..2
  compact      c[m*NAT0 + q] = v[m*NAT + occ[q]], occ = ascending occupied j
  aoff         (a23, a31, a12) per site (``cprod:339-343``)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

try:  # scipy.fft is faster and multi-threaded; numpy.fft is the fallback
    import scipy.fft as _sfft
    from scipy.special import sici as _sici
except Exception:  # pragma: no cover
    _sfft = None
    _sici = None

RELIABLE_RESID_PERIOD = 20      # cu:221
RELIABLE_RESID_GAP = 1.0e-3     # cu:222


# --------------------------------------------------------------------------
# small helpers
# --------------------------------------------------------------------------
def dotc(a, b):
    """sum conj(a)*b in complex128 (cu:260-283 with conjugate=true)."""
    return complex(np.vdot(a.astype(np.complex128, copy=False), b.astype(np.complex128, copy=False)))


def dotu(a, b):
    """sum a*b in complex128 (cu:260-283 with conjugate=false)."""
    return complex(np.dot(a.astype(np.complex128, copy=False), b.astype(np.complex128, copy=False)))


def nrm2(a):
    """FP64 2-norm via the conjugated dot, clipped at 0 (cu:298-307)."""
    v = dotc(a, a).real
    if v < 0.0 and v > -1e-12:
        v = 0.0
    return math.sqrt(max(v, 0.0))


def occupied_index(iocc):
    """Ascending occupied full-grid indices (cu:685-691)."""
    return np.flatnonzero(np.asarray(iocc) != 0).astype(np.int64)


def gather_compact(full, occ, nat):
    """compact[c*NAT0+q] = full[c*NAT+occ[q]] (cu:123-128)."""
    full = np.asarray(full).reshape(3, nat)
    return full[:, occ].reshape(-1)


def scatter_full(compact, occ, nat):
    """full[c*NAT+occ[q]] = compact[c*NAT0+q], zeros elsewhere (cu:129-134, cu:518-522)."""
    nat0 = occ.size
    out = np.zeros((3, nat), dtype=np.asarray(compact).dtype)
    out[:, occ] = np.asarray(compact).reshape(3, nat0)
    return out.reshape(-1)


# --------------------------------------------------------------------------
# Green tensor (cu:600-652)
# --------------------------------------------------------------------------
@dataclass
class GreenParams:
    nx: int
    ny: int
    nz: int
    ipbc: int = 0
    idipint: int = 0
    gamma: float = 0.0
    pyd: float = 0.0
    pzd: float = 0.0
    ak: tuple = (0.0, 0.0, 0.0)
    dx: tuple = (1.0, 1.0, 1.0)

    @property
    def akd(self):
        return math.sqrt(sum(float(a) * float(a) for a in self.ak))


def _cisi(x):
    """Ci and Si for x>0 (the reference uses a continued fraction, cu:610-621;
    here scipy's double-precision routine stands in)."""
    si, ci = _sici(x)
    return ci, si


def green_interaction(x, y, z, akd, idipint, phasyz=0.0, damp=0.0):
    """Six components (xx,xy,xz,yy,yz,zz) of the direct interaction at
    separation (x,y,z); arrays broadcast.  Follows cu:622-633."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    z = np.asarray(z, dtype=np.float64)
    r2 = x * x + y * y + z * z
    ok = r2 > 1.0e-6
    r2s = np.where(ok, r2, 1.0)
    r = np.sqrt(r2s)
    r3 = r * r2s
    kr = akd * r
    xx = (x, y, z)
    out = [np.zeros(np.broadcast(x, y, z).shape, dtype=np.complex128) for _ in range(6)]
    if idipint == 0:
        # point dipole, cu:624-626
        ph = np.exp(1j * (kr + phasyz) - damp) / r3
        fac = (1.0 - 1j * kr) / r2s
        akd2 = akd * akd
        m = 0
        for ii in range(3):
            q = xx[ii] * xx[ii]
            term = akd2 * (q - r2s) + fac * (r2s - 3.0 * q)
            out[m] -= ph * term
            m += 1
            for jj in range(ii + 1, 3):
                term2 = akd2 - 3.0 * fac
                out[m] -= ph * term2 * xx[ii] * xx[jj]
                m += 1
    elif idipint == 1:
        # filtered coupled dipole (FLTRCD), cu:627-631
        pi = math.pi
        kf = pi
        kfr = kf * r
        cip, sip = _cisi(kfr + kr)
        cim, sim = _cisi(np.abs(kfr - kr))
        sim = np.where(kfr - kr < 0.0, -sim, sim)
        sinkr, coskr = np.sin(kr), np.cos(kr)
        sinkfr, coskfr = np.sin(kfr), np.cos(kfr)
        akd2 = akd * akd
        a0 = sinkr * (cip - cim) + coskr * (pi - sip - sim)
        a1 = akd * sinkr * (-pi + sip + sim) + akd * coskr * (cip - cim) - 2.0 * sinkfr / r
        a2 = akd2 * (sinkr * (cim - cip) + coskr * (sip + sim - pi)) + 2.0 * (sinkfr - kfr * coskfr) / r2s
        eikr = np.exp(1j * kr)
        ph = np.exp(1j * phasyz - damp)
        g0 = (eikr - a0 / pi) / r
        g1 = (eikr * (-1.0 + 1j * kr) + (a0 - a1 * r) / pi) / r2s
        g2 = (eikr * (2.0 - kr * kr - 2j * kr) - (2.0 * (a0 - r * a1) + r2s * a2) / pi) / r3
        h2 = (sinkfr - kfr * coskfr) / (pi * r3)
        radial = g2 / r2s - g1 / r3
        m = 0
        for ii in range(3):
            base = g0 * akd2 + g1 / r + (2.0 / 3.0) * h2 + radial * xx[ii] * xx[ii]
            out[m] += ph * base
            m += 1
            for jj in range(ii + 1, 3):
                out[m] += ph * radial * xx[ii] * xx[jj]
                m += 1
    else:
        raise ValueError("idipint must be 0 or 1")
    return [np.where(ok, o, 0.0) for o in out]


def green_lag_grid(p: GreenParams):
    """Direct Green sum on the 2n padded lag grid, lag n planes zeroed
    (cu:634-645, ipbc=0).  Returns array (6, Mz, My, Mx) complex128."""
    if p.ipbc != 0:
        return _green_lag_grid_pbc(p)
    nx, ny, nz = p.nx, p.ny, p.nz
    lx = np.arange(2 * nx)
    ly = np.arange(2 * ny)
    lz = np.arange(2 * nz)
    lx = np.where(lx < nx, lx, lx - 2 * nx)
    ly = np.where(ly < ny, ly, ly - 2 * ny)
    lz = np.where(lz < nz, lz, lz - 2 * nz)
    X = (lx * p.dx[0])[None, None, :]
    Y = (ly * p.dx[1])[None, :, None]
    Z = (lz * p.dx[2])[:, None, None]
    comps = green_interaction(X, Y, Z, p.akd, p.idipint)
    g = np.stack(comps)
    g[:, :, :, nx] = 0.0
    g[:, :, ny, :] = 0.0
    g[:, nz, :, :] = 0.0
    return g


def _green_lag_grid_pbc(p: GreenParams):
    """Periodic-replica Green sum (cu:634-643, ipbc=1).  Small grids only."""
    nx, ny, nz = p.nx, p.ny, p.nz
    akx, aky, akz = (float(a) for a in p.ak)
    akd = p.akd
    akd2 = akd * akd
    pyddx = p.pyd * p.dx[1]
    pzddx = p.pzd * p.dx[2]
    g = np.zeros((6, 2 * nz, 2 * ny, 2 * nx), dtype=np.complex128)
    if pyddx <= 0.0:
        jpbc, kp2 = 2, akx * akx + aky * aky
    elif pzddx <= 0.0:
        jpbc, kp2 = 1, akx * akx + akz * akz
    else:
        jpbc, kp2 = 3, akx * akx
    if kp2 <= 0.0:
        raise ValueError("KPERP: k_perp is zero")
    kperp = math.sqrt(kp2)
    phimax = 1.0 / p.gamma
    term0 = akd2 * phimax * phimax / kp2
    term1 = 2.0 * akd * phimax
    term2y = aky * phimax / kp2
    term2z = akz * phimax / kp2
    beta = 16.0 / phimax ** 4
    for iz in range(2 * nz):
        for iy in range(2 * ny):
            for ix in range(2 * nx):
                if ix == nx or iy == ny or iz == nz:
                    continue
                lx = ix if ix < nx else ix - 2 * nx
                ly = iy if iy < ny else iy - 2 * ny
                lz = iz if iz < nz else iz - 2 * nz
                x0, y0, z0 = lx * p.dx[0], ly * p.dx[1], lz * p.dx[2]
                jpy1 = jpy2 = jpz1 = jpz2 = 0
                if jpbc == 1:
                    rperp = math.sqrt(x0 * x0 + z0 * z0)
                    krf = akd2 * rperp / kperp
                    yf = y0 - aky * rperp / kperp
                    phasf = aky * yf
                    term3 = math.sqrt(term0 + term1 * rperp) / kperp
                    jpy1 = int((yf - term2y - term3) / pyddx + 0.999999)
                    jpy2 = int((yf - term2y + term3) / pyddx)
                elif jpbc == 2:
                    rperp = math.sqrt(x0 * x0 + y0 * y0)
                    krf = akd2 * rperp / kperp
                    zf = z0 - akz * rperp / kperp
                    phasf = akz * zf
                    term3 = math.sqrt(term0 + term1 * rperp) / kperp
                    jpz1 = int((zf - term2z - term3) / pzddx + 0.999999)
                    jpz2 = int((zf - term2z + term3) / pzddx)
                else:
                    rperp = abs(x0)
                    krf = akd2 * rperp / kperp
                    yf = y0 - aky * rperp / kperp
                    zf = z0 - akz * rperp / kperp
                    phasf = aky * yf + akz * zf
                    term3 = math.sqrt(term0 + term1 * rperp) / kperp
                    jpy1 = int((yf - term2y - term3) / pyddx + 0.999999)
                    jpy2 = int((yf - term2y + term3) / pyddx)
                    jpz1 = int((zf - term2z - term3) / pzddx + 0.999999)
                    jpz2 = int((zf - term2z + term3) / pzddx)
                acc = np.zeros(6, dtype=np.complex128)
                for jpy in range(jpy1, jpy2 + 1):
                    rjpy = jpy * pyddx * p.dx[1]
                    yy = y0 - rjpy
                    phasy = aky * rjpy
                    for jpz in range(jpz1, jpz2 + 1):
                        rjpz = jpz * pzddx * p.dx[2]
                        zz = z0 - rjpz
                        r2 = x0 * x0 + yy * yy + zz * zz
                        if r2 <= 1e-6:
                            continue
                        r = math.sqrt(r2)
                        phasyz = phasy + akz * rjpz
                        phi = akd * r - krf + phasyz - phasf
                        damp = beta * phi ** 4
                        c = green_interaction(x0, yy, zz, akd, p.idipint, phasyz, damp)
                        acc += np.array([complex(v) for v in c])
                g[:, iz, iy, ix] = acc
    return g


def _ifftn_unnorm(a, axes):
    """Unnormalised transform with exp(+i) (cuFFT INVERSE convention)."""
    n = 1
    for ax in axes:
        n *= a.shape[ax]
    if _sfft is not None:
        return _sfft.ifftn(a, axes=axes, workers=-1) * n
    return np.fft.ifftn(a, axes=axes) * n


def _fftn(a, axes):
    if _sfft is not None:
        return _sfft.fftn(a, axes=axes, workers=-1)
    return np.fft.fftn(a, axes=axes)


def green_spectrum_full(p: GreenParams):
    """FFT(+i) of the lag grid, all 6 components (cu:649-650)."""
    return _ifftn_unnorm(green_lag_grid(p), axes=(1, 2, 3))


def green_octant(p: GreenParams):
    """The (n+1)^3 octant of the transformed tensor, layout
    g[m][iz][iy][ix] (cu:646, cu:649; the CXZC layout cprod:346-349)."""
    full = green_spectrum_full(p)
    return np.ascontiguousarray(full[:, : p.nz + 1, : p.ny + 1, : p.nx + 1])


def expand_octant(oct6, nx, ny, nz):
    """Rebuild the full (6, Mz, My, Mx) spectrum from the octant with the
    off-diagonal sign rules of cu:112 (s_a = +1 if i_a <= n_a else -1)."""
    Mx, My, Mz = 2 * nx, 2 * ny, 2 * nz
    ix = np.arange(Mx)
    iy = np.arange(My)
    iz = np.arange(Mz)
    irx = np.minimum(ix, Mx - ix)
    iry = np.minimum(iy, My - iy)
    irz = np.minimum(iz, Mz - iz)
    sx = np.where(ix <= nx, 1.0, -1.0)[None, None, :]
    sy = np.where(iy <= ny, 1.0, -1.0)[None, :, None]
    sz = np.where(iz <= nz, 1.0, -1.0)[:, None, None]
    g = oct6[:, irz][:, :, iry][:, :, :, irx]
    sign = [1.0, sx * sy, sx * sz, 1.0, sy * sz, 1.0]
    return np.stack([g[m] * sign[m] for m in range(6)])


# --------------------------------------------------------------------------
# MATVEC (cu:104-118, cu:406-415, cprod:446-607)
# --------------------------------------------------------------------------
class Operator:
    """y = A x for the DDA interaction matrix, FFT-based, FP64 by default.

    ``green_full`` is the (6, Mz, My, Mx) spectrum.  ``apply_full`` mirrors
    ``ddscat_cuda_apply_f32`` (full vectors, unoccupied outputs zeroed,
    unoccupied inputs *not* masked, cu:104-118); ``apply_compact`` mirrors the
    solver MATVEC (``matvec_solver_device``, cu:536-540)."""

    def __init__(self, nx, ny, nz, green_full, iocc, dtype=np.complex128):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nat = nx * ny * nz
        self.iocc = np.asarray(iocc).astype(np.int16)
        self.occ = occupied_index(self.iocc)
        self.nat0 = self.occ.size
        self.dtype = np.dtype(dtype)
        self.green = green_full.astype(self.dtype, copy=False)
        self.ngrid = 8 * self.nat

    @classmethod
    def from_params(cls, p: GreenParams, iocc, dtype=np.complex128):
        return cls(p.nx, p.ny, p.nz, green_spectrum_full(p), iocc, dtype)

    @classmethod
    def from_octant(cls, nx, ny, nz, oct6, iocc, dtype=np.complex128):
        return cls(nx, ny, nz, expand_octant(np.asarray(oct6), nx, ny, nz), iocc, dtype)

    def eself(self, x3):
        """E field from the other dipoles for x of shape (3, nz, ny, nx)."""
        nx, ny, nz = self.nx, self.ny, self.nz
        w = np.zeros((3, 2 * nz, 2 * ny, 2 * nx), dtype=self.dtype)
        w[:, :nz, :ny, :nx] = x3
        w = _ifftn_unnorm(w, axes=(1, 2, 3))
        g = self.green
        px, py, pz = w[0], w[1], w[2]
        out = np.empty_like(w)
        out[0] = g[0] * px + g[1] * py + g[2] * pz
        out[1] = g[1] * px + g[3] * py + g[4] * pz
        out[2] = g[2] * px + g[4] * py + g[5] * pz
        out = _fftn(out, axes=(1, 2, 3))
        return out[:, :nz, :ny, :nx] / float(self.ngrid)

    def apply_full(self, x, adia, aoff, cwhat="N"):
        nat = self.nat
        x = np.asarray(x).astype(self.dtype).reshape(3, nat)
        adia = np.asarray(adia).astype(self.dtype).reshape(3, nat)
        aoff = np.asarray(aoff).astype(self.dtype).reshape(3, nat)
        if cwhat == "C":
            x = np.conj(x)
        w = self.eself(x.reshape(3, self.nz, self.ny, self.nx)).reshape(3, nat)
        y = adia * x - w
        a23, a31, a12 = aoff
        y[0] += a31 * x[2] + a12 * x[1]
        y[1] += a12 * x[0] + a23 * x[2]
        y[2] += a23 * x[1] + a31 * x[0]
        if cwhat == "C":
            y = np.conj(y)
        y[:, self.iocc == 0] = 0.0
        return y.reshape(-1)

    def apply_compact(self, xc, adia_c, aoff_c, cwhat="N"):
        """Compact in, compact out; adia/aoff given compact."""
        nat = self.nat
        xf = scatter_full(xc, self.occ, nat)
        af = scatter_full(adia_c, self.occ, nat)
        of = scatter_full(aoff_c, self.occ, nat)
        y = self.apply_full(xf, af, of, cwhat)
        return gather_compact(y, self.occ, nat)


def dense_matrix(nx, ny, nz, iocc, adia, aoff, akd, idipint=0, dx=(1.0, 1.0, 1.0)):
    """Dense 3NAT x 3NAT matrix of the operator (no FFT) for tiny grids.
    A = diag(adia) + 3x3 site blocks(aoff) - G(r_j - r_k), unoccupied rows 0."""
    nat = nx * ny * nz
    j = np.arange(nat)
    ix, iy, iz = j % nx, (j // nx) % ny, j // (nx * ny)
    DX = (ix[:, None] - ix[None, :]) * dx[0]
    DY = (iy[:, None] - iy[None, :]) * dx[1]
    DZ = (iz[:, None] - iz[None, :]) * dx[2]
    c = green_interaction(DX, DY, DZ, akd, idipint)
    comp = {(0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5}
    A = np.zeros((3 * nat, 3 * nat), dtype=np.complex128)
    for a in range(3):
        for b in range(3):
            m = comp[(min(a, b), max(a, b))]
            A[a * nat:(a + 1) * nat, b * nat:(b + 1) * nat] = -c[m]
    adia = np.asarray(adia, dtype=np.complex128).reshape(3, nat)
    aoff = np.asarray(aoff, dtype=np.complex128).reshape(3, nat)
    for a in range(3):
        A[a * nat + j, a * nat + j] += adia[a]
    a23, a31, a12 = aoff
    A[0 * nat + j, 2 * nat + j] += a31
    A[0 * nat + j, 1 * nat + j] += a12
    A[1 * nat + j, 0 * nat + j] += a12
    A[1 * nat + j, 2 * nat + j] += a23
    A[2 * nat + j, 1 * nat + j] += a23
    A[2 * nat + j, 0 * nat + j] += a31
    dead = np.flatnonzero(np.asarray(iocc) == 0)
    for a in range(3):
        A[a * nat + dead, :] = 0.0
    return A


# --------------------------------------------------------------------------
# Krylov solvers.  Each works on compact vectors with a callback mv(v)
# returning A v (compact), and returns a SolveResult.
# --------------------------------------------------------------------------
@dataclass
class SolveResult:
    x: np.ndarray
    itno: int
    tole: float
    ncompte: int
    status: int = 0
    history: list = field(default_factory=list)


class _Counter:
    def __init__(self, mv):
        self.mv = mv
        self.n = 0

    def __call__(self, v):
        self.n += 1
        return self.mv(v)


def _reliable(mv, rhs, xcur, rrec, rhsnorm, recursive_res, tol):
    """True residual and recursion gap check (cu:543-556)."""
    ax = mv(xcur)
    tr = math.sqrt(max(0.0, float(np.sum(np.abs(rhs.astype(np.complex128) - ax) ** 2))))
    gapn = math.sqrt(max(0.0, float(np.sum(np.abs(rhs.astype(np.complex128) - ax - rrec) ** 2))))
    true_res = tr / rhsnorm
    gap = gapn / tr if tr > 0.0 else (0.0 if gapn == 0.0 else math.inf)
    converged = true_res <= tol
    restart = gap >= RELIABLE_RESID_GAP or (recursive_res <= tol and not converged)
    return ax, true_res, converged, restart


def _c(v):
    return np.asarray(v, dtype=np.complex128).copy()


def solve_pbcgs2(mv, b, x0, maxit, tol):
    """ZBCG2 / BiCGStab(2) with reliable updates, restated from cu:459-480 and
    cu:1168-1278 (including the x0-as-XP convention of cu:462)."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    z = np.zeros(n, dtype=np.complex128)
    rr = b.copy()
    r = [b.copy(), z.copy(), z.copy()]
    u = [z.copy(), z.copy(), z.copy()]
    XP = _c(x0)
    BP = b.copy()
    X = z.copy()
    rnrm0 = nrm2(r[0])
    rnrm = mxnrmx = mxnrmr = rnrm0
    alpha, omega, sigma, rho0 = 0j, 1 + 0j, 1 + 0j, 1 + 0j
    resid = 1.0 if rnrm0 > 0.0 else 0.0
    it = 0
    hist = [resid]
    while resid > tol and it < maxit:
        it += 1
        rho0 = -(omega * rho0)
        for k in (1, 2):
            rho1 = dotc(rr, r[k - 1])
            if rho0 == 0:
                return SolveResult(X, it, resid, mvc.n, 95, hist)
            beta = alpha * (rho1 / rho0)
            rho0 = rho1
            for j in range(k):
                u[j] = r[j] - beta * u[j]
            u[k] = mvc(u[k - 1])
            sigma = dotc(rr, u[k])
            if sigma == 0:
                return SolveResult(X, it, resid, mvc.n, 98, hist)
            alpha = rho1 / sigma
            X = X + alpha * u[0]
            for j in range(k):
                r[j] = r[j] - alpha * u[j + 1]
            r[k] = mvc(r[k - 1])
            rnrm = nrm2(r[0])
            mxnrmx = max(mxnrmx, rnrm)
            mxnrmr = max(mxnrmr, rnrm)
        Z = np.empty((3, 3), dtype=np.complex128)
        for i in range(3):
            for j in range(3):
                Z[i, j] = dotc(r[i], r[j])
        if Z[1, 1] == 0:
            return SolveResult(X, it, resid, mvc.n, 102, hist)
        y0 = np.array([-1.0, Z[1, 0] / Z[1, 1], 0.0], dtype=np.complex128)
        yl = np.array([0.0, Z[1, 2] / Z[1, 1], -1.0], dtype=np.complex128)
        zy0 = Z @ y0
        zyl = Z @ yl
        q0 = np.vdot(y0, zy0)
        ql = np.vdot(yl, zyl)
        k0 = math.sqrt(abs(q0))
        kl = math.sqrt(abs(ql))
        if k0 == 0.0 or kl == 0.0:
            return SolveResult(X, it, resid, mvc.n, 102, hist)
        vr = np.vdot(yl, zy0) / (k0 * kl)
        avr = abs(vr)
        if avr == 0.0:
            return SolveResult(X, it, resid, mvc.n, 102, hist)
        hg = vr * max(avr, 0.7) / avr
        fac = hg * k0 / kl
        y0 = y0 - fac * yl
        Y1, Y2 = y0[1], y0[2]
        omega = y0[2]
        qr = np.vdot(y0, Z @ y0)
        rnrm = math.sqrt(abs(qr))
        mxnrmx = max(mxnrmx, rnrm)
        mxnrmr = max(mxnrmr, rnrm)
        u[0] = u[0] - Y1 * u[1] - Y2 * u[2]
        X = X + Y1 * r[0] + Y2 * r[1]
        r[0] = r[0] - Y1 * r[1] - Y2 * r[2]
        delta = 1.0e-2
        xpdt = rnrm < delta * rnrm0 and rnrm0 < mxnrmx
        rcmp = (rnrm < delta * mxnrmr and rnrm0 < mxnrmr) or xpdt
        resid = rnrm / rnrm0 if rnrm0 > 0.0 else 0.0
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, BP, X, r[0], rnrm0, resid, tol)
            if conv:
                resid = tres
                hist.append(resid)
                break
            if rest:
                r[0] = BP - ax
                XP = X + XP
                X = z.copy()
                BP = r[0].copy()
                rr = r[0].copy()
                for v in (r[1], r[2], u[0], u[1], u[2]):
                    v[:] = 0
                rnrm = mxnrmx = mxnrmr = tres * rnrm0
                alpha, omega, sigma, rho0 = 0j, 1 + 0j, 1 + 0j, 1 + 0j
                resid = tres
                hist.append(resid)
                continue
        if rcmp:
            ax = mvc(X)
            r[0] = BP - ax
            if xpdt:
                XP = X + XP
                X = z.copy()
                BP = r[0].copy()
            mxnrmr = rnrm
            if xpdt:
                mxnrmx = rnrm
        hist.append(resid)
    X = X + XP
    ax = mvc(X)
    rfin = b - ax
    resid = nrm2(rfin) / rnrm0 if rnrm0 > 0 else math.inf
    return SolveResult(X, it, resid, mvc.n, 0, hist)


def solve_qmrccg(mv, b, x0, maxit, tol):
    """Complex-symmetric QMR, restated from cu:434-443 and cu:1071-1103."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    bnorm = nrm2(b)
    if bnorm == 0.0:
        return SolveResult(_c(x0), 0, 0.0, 0, 52)
    xs = _c(x0)
    ax = mvc(xs)
    r = b - ax
    z = np.zeros(n, dtype=np.complex128)
    p, ap, q, d, s = z.copy(), z.copy(), z.copy(), z.copy(), z.copy()
    vt, wt = r.copy(), r.copy()
    sc = {}

    def init_scalars():
        gnorm, knorm = nrm2(vt), nrm2(wt)
        rho = dotu(vt, wt)
        atw = mvc(wt)
        eps = dotu(vt, atw)
        sc.update(lam=1 + 0j, kappa=-1 + 0j, theta=-1 + 0j, gamma=complex(gnorm), ksi=complex(knorm), mu=0j,
                  rho=rho, eps=eps)
        if rho == 0:
            return 5, atw
        if gnorm == 0:
            return 6, atw
        if knorm == 0:
            return 7, atw
        sc["tau"] = eps / rho
        return 0, atw

    st, atw = init_scalars()
    if st:
        return SolveResult(xs, 0, math.inf, mvc.n, 55)
    resid = nrm2(r) / bnorm
    it = 0
    hist = [resid]
    while it < maxit and resid > tol:
        it += 1
        p = vt / sc["gamma"] - sc["mu"] * p
        q = (atw - (sc["gamma"] * sc["mu"]) * q) / sc["ksi"]
        apn = mvc(p)
        ap = apn
        vt = apn - (sc["tau"] / sc["gamma"]) * vt
        wt = q - (sc["tau"] / sc["ksi"]) * wt
        gnorm, knorm = nrm2(vt), nrm2(wt)
        new_rho = dotu(vt, wt)
        atw = mvc(wt)
        new_eps = dotu(vt, atw)
        gamma0, ksi0, rho0, tau0, kappa0 = sc["gamma"], sc["ksi"], sc["rho"], sc["tau"], sc["kappa"]
        gamma, ksi, rho, eps = complex(gnorm), complex(knorm), new_rho, new_eps
        sc.update(gamma=gamma, ksi=ksi, rho=rho, eps=eps)
        if gamma == 0 or ksi == 0:
            return SolveResult(xs, it, resid, mvc.n, 58)
        den = gamma * tau0 * rho0
        if den == 0:
            return SolveResult(xs, it, resid, mvc.n, 58)
        mu = gamma0 * ksi0 * rho / den
        if rho == 0:
            return SolveResult(xs, it, resid, mvc.n, 58)
        tau = eps / rho - gamma * mu
        at0 = abs(tau0) ** 2
        ag = abs(gamma) ** 2
        lam = sc["lam"]
        den2 = lam * at0 + ag
        if den2 == 0:
            return SolveResult(xs, it, resid, mvc.n, 58)
        theta = (1.0 - lam) * at0 / den2
        kappa = -(gamma0 * np.conj(tau0) * kappa0) / den2
        lam = lam * at0 / den2
        sc.update(mu=mu, tau=tau, theta=theta, kappa=kappa, lam=lam)
        d = theta * d + kappa * p
        s = theta * s + kappa * ap
        xs = xs + d
        r = r - s
        resid = nrm2(r) / bnorm
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, b, xs, r, bnorm, resid, tol)
            if conv:
                resid = tres
                hist.append(resid)
                break
            if rest:
                rt = b - ax
                r = rt.copy()
                p, ap, q, d, s = z.copy(), z.copy(), z.copy(), z.copy(), z.copy()
                vt, wt = rt.copy(), rt.copy()
                st, atw = init_scalars()
                if st:
                    return SolveResult(xs, it, resid, mvc.n, 55)
                resid = tres
        hist.append(resid)
    if resid > tol:
        ax, tres, _, _ = _reliable(mvc, b, xs, r, bnorm, resid, tol)
        resid = tres
    return SolveResult(xs, it, resid, mvc.n, 0, hist)


def solve_pbcgst(mv, b, x0, maxit, tol, adia_c):
    """PIM BiCGStab with left DIAGL preconditioning, restart every 5 steps and
    a true residual every iteration, restated from cu:445-457, cu:1105-1165."""
    mvc = _Counter(mv)
    b = _c(b)
    adia_c = _c(adia_c)
    bnorm = nrm2(b)
    xs = _c(x0)
    total_it, converged = 0, False
    resid = 1.0
    hist = [resid]
    while total_it < maxit and not converged:
        ax = mvc(xs)
        rtrue = b - ax
        r = rtrue / adia_c
        rt = r.copy()
        p = np.zeros_like(r)
        v = np.zeros_like(r)
        rho = alpha = omega = 1 + 0j
        for _ in range(5):
            if not (total_it < maxit and not converged):
                break
            new_rho = dotc(rt, r)
            kap = rho * omega
            if kap == 0:
                return SolveResult(xs, total_it, resid, mvc.n, 75, hist)
            beta = new_rho * alpha / kap
            rho = new_rho
            p = r + beta * (p - omega * v)
            v = mvc(p) / adia_c
            xi = dotc(rt, v)
            if xi == 0:
                return SolveResult(xs, total_it, resid, mvc.n, 78, hist)
            alpha = rho / xi
            sv = r - alpha * v
            if nrm2(sv) < 1.19209e-7:
                xs = xs + alpha * p
                total_it += 1
                break
            t = mvc(sv) / adia_c
            tt = dotc(t, t)
            ts = dotc(t, sv)
            if tt == 0:
                return SolveResult(xs, total_it, resid, mvc.n, 82, hist)
            omega = ts / tt
            xs = xs + alpha * p + omega * sv
            r = sv - omega * t
            total_it += 1
            ax = mvc(xs)
            rtrue = b - ax
            resid = nrm2(rtrue) / bnorm if bnorm > 0 else math.inf
            hist.append(resid)
            if resid <= tol:
                converged = True
    if not converged:
        ax = mvc(xs)
        resid = nrm2(b - ax) / bnorm if bnorm > 0 else math.inf
    return SolveResult(xs, total_it, resid, mvc.n, 0 if converged else 87, hist)


def solve_petrkp(mv, mvc_conj, b, x0, maxit, tol):
    """PETR90VER2 CG on the normal equations, restated from cu:482-493 and
    cu:1280-1357.  ``mvc_conj`` applies A^H (the 'C' MATVEC)."""
    cnt = [0]

    def A(v):
        cnt[0] += 1
        return mv(v)

    def AH(v):
        cnt[0] += 1
        return mvc_conj(v)

    b = _c(b)
    xs = _c(x0)
    bb = dotc(b, b).real
    ace = AH(b)
    gi = ace.copy()
    pi = ace.copy()
    qi = A(pi)
    gg = dotc(gi, gi).real
    qq = dotc(qi, qi).real
    if qq == 0.0:
        return SolveResult(xs, 0, math.inf, cnt[0], 115)
    alpha = gg / qq
    xs = xs + alpha * pi
    axi = A(xs)
    resid = 1.0
    hist = [resid]
    it = 1
    while it <= maxit:
        oldgg = gg
        gi = ace - AH(axi)
        gg = dotc(gi, gi).real
        if oldgg == 0.0:
            return SolveResult(xs, it, resid, cnt[0], 119)
        beta = gg / oldgg
        pi = gi + beta * pi
        qi = A(pi)
        qq = dotc(qi, qi).real
        if qq == 0.0:
            return SolveResult(xs, it, resid, cnt[0], 121)
        alpha = gg / qq
        xs = xs + alpha * pi
        if it % 10 != 0:
            axi = axi + alpha * qi
        else:
            axi = A(xs)
        rv = axi - b
        rr = dotc(rv, rv).real
        resid = math.sqrt(max(rr, 0.0) / bb) if bb > 0 else math.inf
        hist.append(resid)
        if resid < tol:
            break
        it += 1
    return SolveResult(xs, min(it, maxit), resid, cnt[0], 0, hist)


def solve_gpbicg(mv, b, x0, maxit, tol):
    """GPBiCG (Zhang), restated from cu:420-432 and cu:1031-1069."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    z0 = np.zeros(n, dtype=np.complex128)
    bnorm = nrm2(b)
    if bnorm == 0.0:
        return SolveResult(_c(x0), 0, 0.0, 0, 32)
    xsol = _c(x0)
    ax = mvc(xsol)
    r0 = b - ax
    r = r0.copy()
    p, t, u, w, zz, y, ap, at, told = (z0.copy() for _ in range(9))
    r0rn = dotc(r0, r0)
    beta = 0j
    resid = nrm2(r) / bnorm
    it = 0
    first = True
    alpha = dz = eta = 0j
    hist = [resid]
    while it < maxit and resid > tol:
        it += 1
        p = r + beta * (p - u)
        ap = mvc(p)
        g0 = dotc(r0, ap)
        if g0 == 0:
            return SolveResult(xsol, it, resid, mvc.n, 34, hist)
        alpha = r0rn / g0
        y = (t - r) + alpha * (ap - w)
        told = t
        t = r - alpha * ap
        at = mvc(t)
        g1 = dotc(at, at)
        g4 = dotc(at, t)
        if first:
            if g1 == 0:
                return SolveResult(xsol, it, resid, mvc.n, 36, hist)
            eta = 0j
            dz = g4 / g1
        else:
            g2 = dotc(y, y)
            g3 = dotc(at, y)
            g5 = dotc(y, t)
            den = g1 * g2 - g3 * np.conj(g3)
            if den == 0:
                return SolveResult(xsol, it, resid, mvc.n, 36, hist)
            dz = (g2 * g4 - g5 * g3) / den
            eta = (g1 * g5 - np.conj(g3) * g4) / den
        unew = dz * ap + eta * ((told - r) + beta * u)
        znew = (dz * r + eta * zz) - alpha * unew
        xsol = xsol + alpha * p + znew
        r = (t - eta * y) - dz * at
        u, zz = unew, znew
        resid = nrm2(r) / bnorm
        hist.append(resid)
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, b, xsol, r, bnorm, resid, tol)
            if conv:
                resid = tres
                break
            if rest:
                rt = b - ax
                r0 = rt.copy()
                r = rt.copy()
                p, y, t, ap, at, u, w, zz, told = (z0.copy() for _ in range(9))
                r0rn = dotc(r0, r0)
                beta = 0j
                first = True
                resid = tres
                continue
        g0 = dotc(r0, r)
        if r0rn == 0 or dz == 0:
            return SolveResult(xsol, it, resid, mvc.n, 39, hist)
        beta = (alpha * g0 / dz) / r0rn
        r0rn = g0
        w = at + beta * ap
        first = False
    if resid > tol:
        ax, tres, _, _ = _reliable(mvc, b, xsol, r, bnorm, resid, tol)
        resid = tres
    return SolveResult(xsol, it, resid, mvc.n, 0, hist)


def solve_bicgstab4(mv, b, x0, maxit, tol):
    """BiCGStab(4) (IFDDA-derived), restated from cu:1363-1433."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    x = _c(x0)
    r = [b - mvc(x)] + [np.zeros(n, dtype=np.complex128) for _ in range(4)]
    u = [np.zeros(n, dtype=np.complex128) for _ in range(5)]
    bnorm, rnorm = nrm2(b), nrm2(r[0])
    if bnorm == 0.0:
        return SolveResult(x, 0, 0.0, mvc.n, 133)
    resid = rnorm / bnorm
    if resid <= tol:
        return SolveResult(x, 0, resid, mvc.n, 0)
    if rnorm < 1e-30:
        return SolveResult(x, 0, resid, mvc.n, 133)
    rtil = r[0] / rnorm
    rho, alpha, omega = 1 + 0j, 0j, 1 + 0j
    hist = [resid]
    it = 1
    while it <= maxit:
        rho = -omega * rho
        for j in range(4):
            if abs(rho) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 135, hist)
            rho1 = dotc(rtil, r[j])
            beta = alpha * rho1 / rho
            rho = rho1
            for i in range(j + 1):
                u[i] = r[i] - beta * u[i]
            u[j + 1] = mvc(u[j])
            den = dotc(rtil, u[j + 1])
            if abs(den) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 137, hist)
            alpha = rho / den
            for i in range(j + 1):
                r[i] = r[i] - alpha * u[i + 1]
            r[j + 1] = mvc(r[j])
            x = x + alpha * u[0]
        tau = np.zeros((4, 4), dtype=np.complex128)
        gp = np.zeros(5, dtype=np.complex128)
        gam = np.zeros(5, dtype=np.complex128)
        gpp = np.zeros(5, dtype=np.complex128)
        sig = np.zeros(5)
        for j in range(1, 5):
            for i in range(1, j):
                tau[j - 1, i - 1] = dotc(r[i], r[j]) / sig[i]
                r[j] = r[j] - tau[j - 1, i - 1] * r[i]
            sig[j] = dotc(r[j], r[j]).real
            if not sig[j] > 1e-30:
                return SolveResult(x, it, resid, mvc.n, 141, hist)
            gp[j] = dotc(r[j], r[0]) / sig[j]
        omega = gam[4] = gp[4]
        for j in range(3, 0, -1):
            gam[j] = gp[j]
            for i in range(j + 1, 5):
                gam[j] -= tau[i - 1, j - 1] * gam[i]
        for j in range(1, 4):
            gpp[j] = gam[j + 1]
            for i in range(j + 1, 4):
                gpp[j] += tau[i - 1, j - 1] * gam[i + 1]
        x = x + gam[1] * r[0]
        r[0] = r[0] - gp[4] * r[4]
        u[0] = u[0] - gam[4] * u[4]
        for j in range(1, 4):
            x = x + gpp[j] * r[j]
            r[0] = r[0] - gp[j] * r[j]
            u[0] = u[0] - gam[j] * u[j]
        rnorm = nrm2(r[0])
        resid = rnorm / bnorm
        hist.append(resid)
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, b, x, r[0], bnorm, resid, tol)
            if conv:
                resid = tres
                break
            if rest:
                r[0] = b - ax
                rnorm = tres * bnorm
                if not rnorm > 0:
                    return SolveResult(x, it, resid, mvc.n, 144, hist)
                rtil = r[0] / rnorm
                u[0] = np.zeros(n, dtype=np.complex128)
                rho, alpha, omega = 1 + 0j, 0j, 1 + 0j
                resid = tres
        it += 1
    ax = mvc(x)
    resid = nrm2(b - ax) / bnorm
    return SolveResult(x, min(it, maxit), resid, mvc.n, 0, hist)


def _solve_small(a, rhs):
    """Partial-pivoting Gaussian elimination with the 1e-30 breakdown test
    of cu:349-359.  Returns None on breakdown."""
    a = np.array(a, dtype=np.complex128)
    bv = np.array(rhs, dtype=np.complex128)
    n = bv.size
    for k in range(n):
        piv = k + int(np.argmax(np.abs(a[k:, k])))
        if abs(a[piv, k]) < 1e-30:
            return None
        if piv != k:
            a[[k, piv], k:] = a[[piv, k], k:]
            bv[[k, piv]] = bv[[piv, k]]
        for i in range(k + 1, n):
            f = a[i, k] / a[k, k]
            a[i, k] = 0
            a[i, k + 1:] -= f * a[k, k + 1:]
            bv[i] -= f * bv[k]
    for i in range(n - 1, -1, -1):
        v = bv[i] - np.dot(a[i, i + 1:], bv[i + 1:])
        if abs(a[i, i]) < 1e-30:
            return None
        bv[i] = v / a[i, i]
    return bv


def solve_gpbicgstab2(mv, b, x0, maxit, tol):
    """GPBiCGStab(2) (IFDDA-derived), restated from cu:1435-1491."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    zv = lambda: np.zeros(n, dtype=np.complex128)  # noqa: E731
    x = _c(x0)
    r0 = b - mvc(x)
    bnorm, rnorm = nrm2(b), nrm2(r0)
    if bnorm == 0.0:
        return SolveResult(x, 0, 0.0, mvc.n, 153)
    rt, p0, z = r0.copy(), r0.copy(), zv()
    yv, u, hs, hq0, hq1, work = zv(), zv(), zv(), zv(), zv(), zv()
    fresh = True
    resid = rnorm / bnorm
    hist = [resid]
    it = 1
    while it <= maxit and resid > tol:
        if fresh:
            rho = dotc(rt, r0)
            work = mvc(p0)
            sigma = dotc(rt, work)
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 154, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            r0 = r0 - alpha * work
            hs = mvc(r0)
            rho = dotc(rt, hs)
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hs - beta * work
            hq1 = mvc(work)
            sigma = dotc(rt, hq1)
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 156, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            r0 = r0 - alpha * work
            hs = hs - alpha * hq1
            hq0 = mvc(hs)
            rho = dotc(rt, hq0)
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hs - beta * work
            hq1 = hq0 - beta * hq1
            mat = np.zeros((2, 2), dtype=np.complex128)
            mat[0, 0] = dotc(hs, hs)
            mat[0, 1] = dotc(hs, hq0)
            mat[1, 1] = dotc(hq0, hq0)
            rhs = np.array([dotc(hs, r0), dotc(hq0, r0)])
            mat[1, 0] = np.conj(mat[0, 1])
            sol = _solve_small(mat, rhs)
            if sol is None:
                return SolveResult(x, it, resid, mvc.n, 159, hist)
            z1, z2 = sol
            z = z1 * r0 + z2 * hs
            x = x + z
            yv = z1 * hs + z2 * hq0
            u = z1 * work + z2 * hq1
            r0 = r0 - yv
            p0 = p0 - u
            hq0 = work.copy()
            fresh = False
        else:
            rho = dotc(rt, r0)
            work = mvc(p0)
            sigma = dotc(rt, work)
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 161, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv + (-alpha) * hq0 + alpha * work
            r0 = r0 - alpha * work
            hs = hs - alpha * hq1
            hq1 = mvc(r0)
            rho = dotc(rt, hq1)
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq1 - beta * work
            hq0 = hs - beta * hq0
            u = yv - beta * u
            hs = mvc(work)
            sigma = dotc(rt, hs)
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 163, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv + (-alpha) * hq0 + alpha * work
            r0 = r0 - alpha * work
            hq1 = hq1 - alpha * hs
            hq0 = mvc(hq1)
            rho = dotc(rt, hq0)
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq1 - beta * work
            hs = hq0 - beta * hs
            u = yv - beta * u
            mat = np.zeros((3, 3), dtype=np.complex128)
            mat[0, 0] = dotc(hq1, hq1)
            mat[0, 1] = dotc(hq1, hq0)
            mat[0, 2] = dotc(hq1, yv)
            mat[1, 1] = dotc(hq0, hq0)
            mat[1, 2] = dotc(hq0, yv)
            mat[2, 2] = dotc(yv, yv)
            rhs = np.array([dotc(hq1, r0), dotc(hq0, r0), dotc(yv, r0)])
            mat[1, 0] = np.conj(mat[0, 1])
            mat[2, 0] = np.conj(mat[0, 2])
            mat[2, 1] = np.conj(mat[1, 2])
            sol = _solve_small(mat, rhs)
            if sol is None:
                return SolveResult(x, it, resid, mvc.n, 166, hist)
            z1, z2, eta = sol
            z = eta * z + z1 * r0 + z2 * hq1
            x = x + z
            yv = eta * yv + z1 * hq1 + z2 * hq0
            u = eta * u + z1 * work + z2 * hs
            r0 = r0 - yv
            p0 = p0 - u
            # restore fixed histories: hs=r1, hq0=p1, hq1=p2 (cu:1474)
            tmp = hs.copy()
            hs = hq1.copy()
            hq1 = tmp
            hq0 = work.copy()
        rnorm = nrm2(r0)
        resid = rnorm / bnorm
        hist.append(resid)
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, b, x, r0, bnorm, resid, tol)
            if conv:
                resid = tres
                break
            if rest:
                r0 = b - ax
                rt, p0, z = r0.copy(), r0.copy(), zv()
                fresh = True
                resid = tres
        it += 1
    if resid > tol:
        ax = mvc(x)
        resid = nrm2(b - ax) / bnorm
    return SolveResult(x, min(it, maxit), resid, mvc.n, 0, hist)


def solve_gpbicgstab4(mv, b, x0, maxit, tol):
    """GPBiCGStab(4) (IFDDA-derived, memory-reduced), restated from
    cu:1493-1570.  Written with explicit polynomial families rr/pp instead of
    the reference's rotating buffer names; the arithmetic is the same."""
    mvc = _Counter(mv)
    b = _c(b)
    n = b.size
    zv = lambda: np.zeros(n, dtype=np.complex128)  # noqa: E731
    x = _c(x0)
    r0 = b - mvc(x)
    bnorm, rnorm = nrm2(b), nrm2(r0)
    if bnorm == 0.0:
        return SolveResult(x, 0, 0.0, mvc.n, 183)
    rt, p0, z = r0.copy(), r0.copy(), zv()
    yv, u = zv(), zv()
    hs = [zv(), zv(), zv()]
    hq = [zv(), zv(), zv(), zv()]
    work = zv()
    fresh = True
    resid = rnorm / bnorm
    hist = [resid]

    def restore():
        nonlocal work
        hq[0] = hs[0].copy(); hs[0] = hq[3].copy(); hq[3] = hq[0].copy()
        hq[0] = hs[1].copy(); hs[1] = hq[2].copy(); hq[2] = hq[0].copy()
        hq[0] = hs[2].copy(); hs[2] = hq[1].copy(); hq[1] = hq[0].copy(); hq[0] = work.copy()

    it = 1
    while it <= maxit and resid > tol:
        if fresh:
            rr = [r0, hq[3], hq[2], hq[1], hq[0]]
            pp = [p0, work, hs[2], hs[1], hs[0]]
            rho = dotc(rt, rr[0])
            for j in range(1, 5):
                pp[j] = mvc(pp[j - 1])
                sigma = dotc(rt, pp[j])
                if abs(sigma) < 1e-30:
                    return SolveResult(x, it, resid, mvc.n, 184, hist)
                alpha = rho / sigma
                x = x + alpha * pp[0]
                for i in range(j):
                    rr[i] = rr[i] - alpha * pp[i + 1]
                rr[j] = mvc(rr[j - 1])
                rho = dotc(rt, rr[j])
                beta = rho / sigma
                for i in range(j + 1):
                    pp[i] = rr[i] - beta * pp[i]
            mat = np.zeros((4, 4), dtype=np.complex128)
            rhs = np.zeros(4, dtype=np.complex128)
            for i in range(4):
                for j in range(4):
                    mat[i, j] = dotc(rr[i + 1], rr[j + 1])
                rhs[i] = dotc(rr[i + 1], rr[0])
            sol = _solve_small(mat, rhs)
            if sol is None:
                return SolveResult(x, it, resid, mvc.n, 187, hist)
            zeta = sol
            z = zeta[0] * rr[0]
            for i in range(1, 4):
                z = z + zeta[i] * rr[i]
            x = x + z
            yv = zeta[0] * rr[1]
            u = zeta[0] * pp[1]
            for i in range(1, 4):
                yv = yv + zeta[i] * rr[i + 1]
                u = u + zeta[i] * pp[i + 1]
            r0 = rr[0] - yv
            p0 = pp[0] - u
            hq[3], hq[2], hq[1], hq[0] = rr[1], rr[2], rr[3], rr[4]
            work, hs[2], hs[1], hs[0] = pp[1], pp[2], pp[3], pp[4]
            restore()
            fresh = False
        else:
            rho = dotc(rt, r0)
            # j=1
            work = mvc(p0)
            sigma = dotc(rt, work)
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 190, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv - alpha * hq[0] + alpha * work
            r0 = r0 - alpha * work
            for i in range(3):
                hs[i] = hs[i] - alpha * hq[i + 1]
            hq[3] = mvc(r0)
            rho = dotc(rt, hq[3])
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq[3] - beta * work
            for i in range(3):
                hq[i] = hs[i] - beta * hq[i]
            u = yv - beta * u
            # j=2
            hs[2] = mvc(work)
            sigma = dotc(rt, hs[2])
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 193, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv - alpha * hq[0] + alpha * work
            r0 = r0 - alpha * work
            hq[3] = hq[3] - alpha * hs[2]
            for i in range(2):
                hs[i] = hs[i] - alpha * hq[i + 1]
            hq[2] = mvc(hq[3])
            rho = dotc(rt, hq[2])
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq[3] - beta * work
            hs[2] = hq[2] - beta * hs[2]
            for i in range(2):
                hq[i] = hs[i] - beta * hq[i]
            u = yv - beta * u
            # j=3
            hs[1] = mvc(hs[2])
            sigma = dotc(rt, hs[1])
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 196, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv - alpha * hq[0] + alpha * work
            r0 = r0 - alpha * work
            hq[3] = hq[3] - alpha * hs[2]
            hq[2] = hq[2] - alpha * hs[1]
            hs[0] = hs[0] - alpha * hq[1]
            hq[1] = mvc(hq[2])
            rho = dotc(rt, hq[1])
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq[3] - beta * work
            hs[2] = hq[2] - beta * hs[2]
            hs[1] = hq[1] - beta * hs[1]
            hq[0] = hs[0] - beta * hq[0]
            u = yv - beta * u
            # j=4
            hs[0] = mvc(hs[1])
            sigma = dotc(rt, hs[0])
            if abs(sigma) < 1e-30:
                return SolveResult(x, it, resid, mvc.n, 199, hist)
            alpha = rho / sigma
            x = x + alpha * p0
            z = z - alpha * u
            yv = yv - alpha * hq[0] + alpha * work
            r0 = r0 - alpha * work
            hq[3] = hq[3] - alpha * hs[2]
            hq[2] = hq[2] - alpha * hs[1]
            hq[1] = hq[1] - alpha * hs[0]
            hq[0] = mvc(hq[1])
            rho = dotc(rt, hq[0])
            beta = rho / sigma
            p0 = r0 - beta * p0
            work = hq[3] - beta * work
            hs[2] = hq[2] - beta * hs[2]
            hs[1] = hq[1] - beta * hs[1]
            hs[0] = hq[0] - beta * hs[0]
            u = yv - beta * u
            rr = [r0, hq[3], hq[2], hq[1], hq[0]]
            pp = [p0, work, hs[2], hs[1], hs[0]]
            mat = np.zeros((5, 5), dtype=np.complex128)
            rhs = np.zeros(5, dtype=np.complex128)
            for i in range(4):
                for j in range(4):
                    mat[i, j] = dotc(rr[i + 1], rr[j + 1])
                mat[i, 4] = dotc(rr[i + 1], yv)
                mat[4, i] = np.conj(mat[i, 4])
                rhs[i] = dotc(rr[i + 1], rr[0])
            mat[4, 4] = dotc(yv, yv)
            rhs[4] = dotc(yv, rr[0])
            sol = _solve_small(mat, rhs)
            if sol is None:
                return SolveResult(x, it, resid, mvc.n, 202, hist)
            zeta, eta = sol[:4], sol[4]
            z = eta * z
            for i in range(4):
                z = z + zeta[i] * rr[i]
            x = x + z
            yv = eta * yv
            u = eta * u
            for i in range(4):
                yv = yv + zeta[i] * rr[i + 1]
                u = u + zeta[i] * pp[i + 1]
            r0 = r0 - yv
            p0 = p0 - u
            restore()
        rnorm = nrm2(r0)
        resid = rnorm / bnorm
        hist.append(resid)
        if it % RELIABLE_RESID_PERIOD == 0 or resid <= tol:
            ax, tres, conv, rest = _reliable(mvc, b, x, r0, bnorm, resid, tol)
            if conv:
                resid = tres
                break
            if rest:
                r0 = b - ax
                rt, p0, z = r0.copy(), r0.copy(), zv()
                fresh = True
                resid = tres
            else:
                work = hq[0].copy()
        it += 1
    ax = mvc(x)
    resid = nrm2(b - ax) / bnorm
    return SolveResult(x, min(it, maxit), resid, mvc.n, 0, hist)


SOLVERS = {
    "pbcgs2": solve_pbcgs2,
    "qmrccg": solve_qmrccg,
    "gpbicg": solve_gpbicg,
    "bicgstab4": solve_bicgstab4,
    "gpbicgstab2": solve_gpbicgstab2,
    "gpbicgstab4": solve_gpbicgstab4,
}


# --------------------------------------------------------------------------
# EVALQ (cu:770-783, cu:919-955)
# --------------------------------------------------------------------------
def evalq(e_c, p_c, adia_c, aoff_c, ak, e02):
    """Cabs, Cext, Cpha from compact E, P, adia, aoff (cu:939-950)."""
    nat0 = np.asarray(p_c).size // 3
    p = np.asarray(p_c, dtype=np.complex128).reshape(3, nat0)
    e = np.asarray(e_c, dtype=np.complex128).reshape(3, nat0)
    ad = np.asarray(adia_c, dtype=np.complex128).reshape(3, nat0)
    ao = np.asarray(aoff_c, dtype=np.complex128).reshape(3, nat0)
    akk = math.sqrt(sum(float(a) ** 2 for a in ak))
    ak3 = akk ** 3
    ri = 1j * (ak3 / 1.5)
    a23, a31, a12 = ao
    q = np.empty_like(p)
    q[0] = (ad[0] + ri) * p[0] + a31 * p[2] + a12 * p[1]
    q[1] = (ad[1] + ri) * p[1] + a12 * p[0] + a23 * p[2]
    q[2] = (ad[2] + ri) * p[2] + a23 * p[1] + a31 * p[0]
    zabs = np.vdot(p.reshape(-1), q.reshape(-1))
    zep = np.vdot(e.reshape(-1), p.reshape(-1))
    cabs = -4.0 * math.pi * akk * zabs.imag / e02
    cext = 4.0 * math.pi * akk * zep.imag / e02
    cpha = 2.0 * math.pi * akk * zep.real / e02
    return cabs, cext, cpha


# --------------------------------------------------------------------------
# SCAT (cu:785-910, cu:957-1002)
# --------------------------------------------------------------------------
def _llround(v):
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))


def scat_integration_dirs(ak, e01, etasca, nat0):
    """(theta,phi) quadrature of cu:849-875.  Returns (dirs float32 (N,3),
    weights float64 (N,5))."""
    pi = 4.0 * math.atan(1.0)
    ak = [float(np.float32(a)) for a in ak]
    ak2 = ak[0] * ak[0] + ak[1] * ak[1] + ak[2] * ak[2]
    akk = math.sqrt(ak2)
    a1 = [float(np.float32(np.real(e))) for e in e01]
    einc = math.sqrt(sum(a * a for a in a1))
    if not einc > 0.0:
        raise ValueError("CXE01_TF is pure imaginary")
    a1 = [a * akk / einc for a in a1]
    a2 = [(ak[1] * a1[2] - ak[2] * a1[1]) / akk,
          (ak[2] * a1[0] - ak[0] * a1[2]) / akk,
          (ak[0] * a1[1] - ak[1] * a1[0]) / akk]
    x = akk * (3.0 * nat0 / (4.0 * pi)) ** (1.0 / 3.0)
    theta0 = 2.0 * pi / (1.0 + x)
    afac = 1.0
    ntheta = 1 + _llround((2.0 * (3.0 + x) / float(np.float32(etasca))) * (1.0 + afac / (pi + theta0))
                          / (1.0 + afac * theta0 / ((pi + theta0) ** 2)))
    theta = thetau = 0.0
    dirs, wts = [], []
    for ic in range(1, ntheta + 1):
        thetal = theta
        theta = thetau
        if ic < ntheta:
            si = ic * (pi + afac * pi / (theta0 + pi)) / (ntheta - 1)
            term = si - afac - theta0
            thetau = 0.5 * (term + math.sqrt(term * term + 4.0 * theta0 * si))
        else:
            thetau = pi
        domega = 2.0 * pi * (math.cos(0.5 * (thetal + theta)) - math.cos(0.5 * (theta + thetau)))
        ct, st = math.cos(theta), math.sin(theta)
        if ic == 1 or ic == ntheta:
            nphi = 1
        else:
            nphi = _llround(4.0 * pi * st / (thetau - thetal))
            if nphi < 3:
                nphi = 3
        w = domega / nphi
        dphi = 2.0 * pi / nphi
        for ip in range(1, nphi + 1):
            phi = dphi * (ip - 0.5 * (ic % 2))
            sp, cp = math.sin(phi), math.cos(phi)
            dirs.append([ct * ak[k] + st * (cp * a1[k] + sp * a2[k]) for k in range(3)])
            wts.append([w, w * ct, w * st * cp, w * st * sp, w * ct * ct])
    return np.asarray(dirs, dtype=np.float32), np.asarray(wts, dtype=np.float64)


def farfield_sums(p_c, occ, nx, ny, dirs, dx, x0):
    """S(dir) = sum_j P_j exp(-i k_s . r_j), r_j = ((i+1)+x0)*dx (cu:793-822).
    FP64 throughout.  Returns (ndir, 3) complex128."""
    nat0 = occ.size
    p = np.asarray(p_c, dtype=np.complex128).reshape(3, nat0)
    ix = occ % nx
    iy = (occ // nx) % ny
    iz = occ // (nx * ny)
    r = np.stack([(ix + 1 + float(x0[0])) * float(dx[0]),
                  (iy + 1 + float(x0[1])) * float(dx[1]),
                  (iz + 1 + float(x0[2])) * float(dx[2])], axis=1)
    out = np.empty((len(dirs), 3), dtype=np.complex128)
    chunk = max(1, 2_000_000 // max(nat0, 1))
    d64 = np.asarray(dirs, dtype=np.float64)
    for s in range(0, len(dirs), chunk):
        ph = np.exp(-1j * (d64[s:s + chunk] @ r.T))
        out[s:s + chunk] = ph @ p.T
    return out


def scat(p_c, occ, nx, ny, jpbc, ak, aks, dx, em1, em2, e02, etasca, e01, x0):
    """Restates ddscat_cuda_scat_f32 (cu:957-1002).  Returns dict with
    cbksca, csca, cscag(3), cscag2, navg, f1, f2."""
    nat0 = occ.size
    ak = [float(np.float32(a)) for a in ak]
    ak2 = sum(a * a for a in ak)
    akk = math.sqrt(ak2)
    ak3 = akk * ak2
    out = {"cbksca": 0.0, "csca": 0.0, "cscag": [0.0, 0.0, 0.0], "cscag2": 0.0, "navg": 0}
    if jpbc == 0:
        dirs, w = scat_integration_dirs(ak, e01, etasca, nat0)
        s = farfield_sums(p_c, occ, nx, ny, dirs, dx, x0)
        n = dirs.astype(np.float64) / akk
        ndp = np.sum(n * s, axis=1)
        e = s - n * ndp[:, None]
        es2 = np.sum(np.abs(e) ** 2, axis=1)
        acc = es2 @ w
        fac = ak2 * ak2 / e02
        out.update(navg=len(dirs), csca=fac * acc[0], cscag=[fac * acc[1], fac * acc[2], fac * acc[3]],
                   cscag2=fac * acc[4], cbksca=fac * es2[-1])
    aks = np.asarray(aks, dtype=np.float32).reshape(-1, 3)
    if aks.shape[0] > 0:
        s = farfield_sums(p_c, occ, nx, ny, aks, dx, x0)
        term = ak3 / math.sqrt(e02)
        em1 = np.asarray(em1, dtype=np.float64).reshape(-1, 3)
        em2 = np.asarray(em2, dtype=np.float64).reshape(-1, 3)
        out["f1"] = term * np.sum(em1 * s, axis=1)
        out["f2"] = term * np.sum(em2 * s, axis=1)
    return out


# --------------------------------------------------------------------------
# Radiative torque (DDSCAT's CMDTRQ = 'DOTORQ' branch of SCAT,
# getfml_cuda.f90:1135-1144; DDSCAT's own SCAT torque sums are not vendored in
# the reference, so this restates the physics from first principles).
#
# Units as in EVALQ/SCAT: P in the solver's normalisation (A P = E), the torque
# reported as a cross section C = 8 pi k Gamma / E02 (Q = C / (pi a_eff^2) is
# DDSCAT's Q_Gamma = Gamma / (pi a_eff^2 u_rad / k) with u_rad = E02 / 8 pi).
#   incident part  Gamma_inc = sum_j 1/2 Re(P_j x E_j*) + r_j x (k/2) Im(P_j . E_j*)
#                  (time-averaged torque of the incident plane wave on the
#                  induced dipoles: the angular momentum it loses, whose
#                  momentum counterpart is C_ext k-hat)
#   scattered flux L_sca = 1/(8 pi k) Int dOmega Im[F_a* (n x grad_n) F_a + F* x F]
#                  with F = k^2 (S - n (n.S)), S = sum_j P_j exp(-i k n.r_j):
#                  (n x grad_n) F_a expands to -i k n x U_a . and -(n x F*)(n.S)
#                  terms, U_ab = sum_j P_ja r_jb exp(-i k n.r_j)
#   net torque     C_net = C_inc - C_flux
# r_j as in SCAT: ((i+1) + x0) * dx.  The angular integration uses SCAT's
# ETASCA quadrature (scat_integration_dirs, first weight column).
# --------------------------------------------------------------------------
def site_positions(occ, nx, ny, dx, x0):
    ix = occ % nx
    iy = (occ // nx) % ny
    iz = occ // (nx * ny)
    return np.stack([(ix + 1 + float(x0[0])) * float(dx[0]),
                     (iy + 1 + float(x0[1])) * float(dx[1]),
                     (iz + 1 + float(x0[2])) * float(dx[2])], axis=1)


def torque_incident(p_c, e_c, r, ak, e02):
    """C_inc (3,) of the incident field E (compact) on the dipoles P at r."""
    nat0 = r.shape[0]
    p = np.asarray(p_c, dtype=np.complex128).reshape(3, nat0).T
    e = np.asarray(e_c, dtype=np.complex128).reshape(3, nat0).T
    ak = np.asarray([float(a) for a in ak])
    akk = float(np.linalg.norm(ak))
    spin = 0.5 * np.real(np.cross(p, np.conj(e))).sum(axis=0)
    w = 0.5 * np.imag(np.sum(p * np.conj(e), axis=1))
    orb = (np.cross(r, ak[None, :]) * w[:, None]).sum(axis=0)
    return 8.0 * math.pi * akk * (spin + orb) / e02


def torque_flux_sums(p_c, r, dirs):
    """S (ndir,3) and U (ndir,3,3), U[:,a,b] = sum_j P_ja r_jb exp(-i k_s . r_j)."""
    nat0 = r.shape[0]
    p = np.asarray(p_c, dtype=np.complex128).reshape(3, nat0).T
    d64 = np.asarray(dirs, dtype=np.float64)
    S = np.empty((len(d64), 3), dtype=np.complex128)
    U = np.empty((len(d64), 3, 3), dtype=np.complex128)
    pr = (p[:, :, None] * r[:, None, :]).reshape(nat0, 9)
    chunk = max(1, 2_000_000 // max(nat0, 1))
    for s in range(0, len(d64), chunk):
        ph = np.exp(-1j * (d64[s:s + chunk] @ r.T))
        S[s:s + chunk] = ph @ p
        U[s:s + chunk] = (ph @ pr).reshape(-1, 3, 3)
    return S, U


def torque_flux_integrand(n, S, U, akk):
    """Im[-i k n x V - (n.S)(n x e*) + e* x e] per direction, e = S - n(n.S),
    V_b = sum_a e_a* U_ab (the bracket of L_sca without the k^4 factor)."""
    nS = np.sum(n * S, axis=1)
    e = S - n * nS[:, None]
    V = np.einsum("da,dab->db", np.conj(e), U)
    val = -1j * akk * np.cross(n, V) - nS[:, None] * np.cross(n, np.conj(e)) + np.cross(np.conj(e), e)
    return np.imag(val)


def scat_torque(p_c, e_c, occ, nx, ny, ak, dx, e02, etasca, e01, x0):
    """Torque cross sections of the resident solution: dict with ctrq_inc (3),
    ctrq_flux (3), ctrq (3) = inc - flux, navg."""
    nat0 = occ.size
    ak = [float(np.float32(a)) for a in ak]
    akk = math.sqrt(sum(a * a for a in ak))
    r = site_positions(occ, nx, ny, dx, x0)
    cinc = torque_incident(p_c, e_c, r, ak, e02)
    dirs, w = scat_integration_dirs(ak, e01, etasca, nat0)
    S, U = torque_flux_sums(p_c, r, dirs)
    n = dirs.astype(np.float64) / akk
    f = torque_flux_integrand(n, S, U, akk)
    cflux = akk ** 4 / e02 * (w[:, 0] @ f)
    return {"ctrq_inc": cinc, "ctrq_flux": cflux, "ctrq": cinc - cflux, "navg": len(dirs)}


# --------------------------------------------------------------------------
# Amplitude and Mueller matrices (the S_ij step DDSCAT's GETMUELLER performs
# after SCAT; GETMUELLER itself is not in the reference).  Restated from the
# definitions of Bohren & Huffman (1983), "Absorption and Scattering of Light by
# Small Particles", section 3.2 (amplitude matrix) and eq. 3.16 (Mueller
# matrix), with DDSCAT's f_ml as the reference SCAT returns them: f_ml is the
# amplitude along the scattered basis vector e_m (m = 1: EM1, m = 2: EM2) for
# incident polarisation e0l (l = 1: E01, l = 2: E02), in the normalisation of
# ddscat_cuda_scat_f32 (term = |k|^3/sqrt(E02), cu:994), i.e. k times the
# physical scattering amplitude, so that S = -i f.

def amplitude_matrix(ak, e01, e02, em2, f11, f21, f12, f22):
    """S1..S4 per direction (ndir, 4) complex128, in the order (S1, S2, S3, S4).

    EM1/EM2 are DDSCAT's scattered basis vectors as passed to SCAT, with
    EM2 = n x EM1 (theta-hat and phi-hat).  Bohren & Huffman use e_par,s =
    theta-hat and e_perp,s = -phi-hat = -EM2, and the same perpendicular vector
    for the incident light, e_perp,i = -EM2, with e_par,i = khat x e_perp,i.
    With a_l = conj(e0l) . E_inc the scattered field components are
    E_par = sum_l f_1l a_l and E_perp = -sum_l f_2l a_l, so with g_1l = f_1l,
    g_2l = -f_2l:
      S2 = -i sum_l g_1l conj(e0l).e_par,i   S3 = -i sum_l g_1l conj(e0l).e_perp,i
      S4 = -i sum_l g_2l conj(e0l).e_par,i   S1 = -i sum_l g_2l conj(e0l).e_perp,i
    """
    k = np.asarray(ak, dtype=np.float64)
    khat = k / np.linalg.norm(k)
    eperp = -np.asarray(em2, dtype=np.float64).reshape(-1, 3)
    epar = np.cross(khat[None, :], eperp)
    e0 = [np.conj(np.asarray(e01, dtype=np.complex128)), np.conj(np.asarray(e02, dtype=np.complex128))]
    cpar = [epar @ e for e in e0]     # conj(e0l) . e_par,i
    cperp = [eperp @ e for e in e0]   # conj(e0l) . e_perp,i
    g1 = [np.asarray(f11, dtype=np.complex128), np.asarray(f12, dtype=np.complex128)]    # l = 1, 2
    g2 = [-np.asarray(f21, dtype=np.complex128), -np.asarray(f22, dtype=np.complex128)]
    S2 = -1j * (g1[0] * cpar[0] + g1[1] * cpar[1])
    S3 = -1j * (g1[0] * cperp[0] + g1[1] * cperp[1])
    S4 = -1j * (g2[0] * cpar[0] + g2[1] * cpar[1])
    S1 = -1j * (g2[0] * cperp[0] + g2[1] * cperp[1])
    return np.stack([S1, S2, S3, S4], axis=1)


def mueller_from_amplitude(S):
    """(ndir, 4, 4) Mueller matrix S_ij from (S1, S2, S3, S4), Bohren & Huffman eq. 3.16."""
    S1, S2, S3, S4 = (S[:, k] for k in range(4))
    a1, a2, a3, a4 = (np.abs(s) ** 2 for s in (S1, S2, S3, S4))
    M = np.empty((S.shape[0], 4, 4))
    M[:, 0, 0] = 0.5 * (a2 + a1 + a4 + a3)
    M[:, 0, 1] = 0.5 * (a2 - a1 + a4 - a3)
    M[:, 0, 2] = np.real(S2 * np.conj(S3) + S1 * np.conj(S4))
    M[:, 0, 3] = np.imag(S2 * np.conj(S3) - S1 * np.conj(S4))
    M[:, 1, 0] = 0.5 * (a2 - a1 - a4 + a3)
    M[:, 1, 1] = 0.5 * (a2 + a1 - a4 - a3)
    M[:, 1, 2] = np.real(S2 * np.conj(S3) - S1 * np.conj(S4))
    M[:, 1, 3] = np.imag(S2 * np.conj(S3) + S1 * np.conj(S4))
    M[:, 2, 0] = np.real(S2 * np.conj(S4) + S1 * np.conj(S3))
    M[:, 2, 1] = np.real(S2 * np.conj(S4) - S1 * np.conj(S3))
    M[:, 2, 2] = np.real(S1 * np.conj(S2) + S3 * np.conj(S4))
    M[:, 2, 3] = np.imag(S2 * np.conj(S1) + S4 * np.conj(S3))
    M[:, 3, 0] = np.imag(S4 * np.conj(S2) + S1 * np.conj(S3))
    M[:, 3, 1] = np.imag(S4 * np.conj(S2) - S1 * np.conj(S3))
    M[:, 3, 2] = np.imag(S1 * np.conj(S2) - S3 * np.conj(S4))
    M[:, 3, 3] = np.real(S1 * np.conj(S2) - S3 * np.conj(S4))
    return M
