"""Seeded synthetic DDA problems (harness code, not the solve path).

The reference takes the target occupancy (TARELL), the incident field (EVALE)
and the polarisabilities (ALPHADIAG/EVALA) from upstream DDSCAT routines that
are not part of it.  This module restates them from published formulas so
tests and the benchmark can build inputs with the shapes of the DDSCAT
configurations:

* occupancy: site (i,j,k) is occupied iff sum_a ((i_a + 1/2 - n_a/2)/r_a)^2 <= 1
  (r_a = semi-axes in lattice units);
* polarisabilities (CXADIA = 1/alpha per Cartesian component, lattice units
  d = 1, alpha_CM = (3/4pi)(m^2-1)/(m^2+2), a = unit propagation vector,
  e = unit polarisation vector), DDSCAT's CMDPOL choices:
  - LATTDR, the lattice dispersion relation of Draine & Goodman (1993, ApJ 405,
    685): 1/alpha = 1/alpha_CM + (b1 + m^2 b2 + m^2 b3 S)(kd)^2 - (2/3) i (kd)^3,
    S = sum_j (a_j e_j)^2, b1 = -1.891531, b2 = 0.1648469, b3 = -1.7700004, the
    same for the three components;
  - GKDLDR, the corrected lattice dispersion relation of Gutkowicz-Krusin &
    Draine (2004, arXiv:astro-ph/0403082): a diagonal tensor whose component j
    has S replaced by a_j^2, so it depends on the direction of propagation but
    not on the polarisation: 1/alpha_jj = 1/alpha_CM + (b1 + m^2 b2 +
    m^2 b3 a_j^2)(kd)^2 - (2/3) i (kd)^3 (the prescription of the synthetic
    workloads, as in DDSCAT's own parameter files);
  - FLTRCD, the filtered coupled dipole polarisability (Piller & Martin 1998;
    Gay-Balmaz & Martin 2002; Yurkin, Min & Hoekstra 2010): 1/alpha =
    1/alpha_CM - (4/3)(kd)^2 - (2/(3 pi)) ln((pi - kd)/(pi + kd)) (kd)^3
    - (2/3) i (kd)^3, for kd < pi;
* incident field E_j = e0 exp(i k.r_j), r_j = ((i+1)+x0)*d, x0 = -(n+1)/2
  (target centred at the origin).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

B1, B2, B3 = -1.891531, 0.1648469, -1.7700004
PRESCRIPTIONS = ("LATTDR", "GKDLDR", "FLTRCD")


def ellipsoid_occupancy(nx, ny, nz, semi=None):
    """int16 IOCC of length nx*ny*nz (component order j = ix + nx*(iy + ny*iz))."""
    if semi is None:
        semi = (nx / 2.0, ny / 2.0, nz / 2.0)
    ix = (np.arange(nx) + 0.5 - nx / 2.0) / semi[0]
    iy = (np.arange(ny) + 0.5 - ny / 2.0) / semi[1]
    iz = (np.arange(nz) + 0.5 - nz / 2.0) / semi[2]
    r2 = iz[:, None, None] ** 2 + iy[None, :, None] ** 2 + ix[None, None, :] ** 2
    return (r2 <= 1.0).astype(np.int16).reshape(-1)


def ldr_alpha(m, kd, khat, ehat):
    """LDR polarisability (lattice units d=1) for refractive index m."""
    eps = complex(m) ** 2
    acm = (3.0 / (4.0 * math.pi)) * (eps - 1.0) / (eps + 2.0)
    S = float(np.sum((np.asarray(khat) * np.real(np.asarray(ehat))) ** 2))
    corr = (B1 + eps * B2 + eps * B3 * S) * kd ** 2 - (2.0 / 3.0) * 1j * kd ** 3
    return acm / (1.0 + acm * corr)


def _shape_factor(khat, ehat, cmdpol):
    """The (kd)^2 term's S per Cartesian component (3,): LATTDR's sum_j (a_j e_j)^2
    for all three, GKDLDR's a_j^2; None for FLTRCD."""
    a = np.asarray(khat, dtype=np.float64)
    if cmdpol == "LATTDR":
        return np.full(3, float(np.sum((a * np.real(np.asarray(ehat))) ** 2)))
    if cmdpol == "GKDLDR":
        return a ** 2
    if cmdpol == "FLTRCD":
        return None
    raise ValueError(f"unknown polarisability prescription {cmdpol!r} (one of {PRESCRIPTIONS})")


def inv_alpha_eps(eps, kd, khat, ehat, cmdpol="GKDLDR"):
    """1/alpha (lattice units) per Cartesian component for permittivity eps
    (scalar or array): shape (3,) + eps.shape."""
    eps = np.asarray(eps, dtype=np.complex128)
    base = (4.0 * math.pi / 3.0) * (eps + 2.0) / (eps - 1.0) - (2.0 / 3.0) * 1j * kd ** 3
    S = _shape_factor(khat, ehat, cmdpol)
    if S is None:
        if not kd < math.pi:
            raise ValueError("FLTRCD needs kd < pi")
        corr = -(4.0 / 3.0) * kd ** 2 - (2.0 / (3.0 * math.pi)) * math.log((math.pi - kd) / (math.pi + kd)) * kd ** 3
        return np.stack([base + corr] * 3)
    return np.stack([base + (B1 + eps * B2 + eps * B3 * S[j]) * kd ** 2 for j in range(3)])


def dinv_alpha_deps(eps, kd, khat, ehat, cmdpol="GKDLDR"):
    """d(1/alpha)/d eps per Cartesian component: shape (3,) + eps.shape."""
    eps = np.asarray(eps, dtype=np.complex128)
    base = -4.0 * math.pi / (eps - 1.0) ** 2
    S = _shape_factor(khat, ehat, cmdpol)
    if S is None:
        return np.stack([base] * 3)
    return np.stack([base + (B2 + B3 * S[j]) * kd ** 2 for j in range(3)])


def euler_rotation(beta, theta, phi):
    """Rotation R = Rz(phi) Ry(theta) Rz(beta) (ZYZ Euler angles)."""
    def rz(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])

    def ry(a):
        c, s = math.cos(a), math.sin(a)
        return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])

    return rz(phi) @ ry(theta) @ rz(beta)


def random_orientations(count, seed=0):
    """Euler angles uniform on SO(3): beta, phi ~ U[0,2pi), cos(theta) ~ U[-1,1]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        beta = rng.uniform(0.0, 2.0 * math.pi)
        ct = rng.uniform(-1.0, 1.0)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        out.append((beta, math.acos(ct), phi))
    return out


@dataclass
class Incidence:
    """One right-hand side: wave vector k (lattice units) and polarisation e."""
    k: np.ndarray
    e: np.ndarray


@dataclass
class Problem:
    nx: int
    ny: int
    nz: int
    iocc: np.ndarray
    m: complex
    kd: float
    aeff: float
    x0: tuple
    incid: list = field(default_factory=list)
    cmdpol: str = "GKDLDR"

    @property
    def nat(self):
        return self.nx * self.ny * self.nz

    @property
    def nat0(self):
        return int(np.count_nonzero(self.iocc))

    @property
    def occ(self):
        return np.flatnonzero(self.iocc)

    def positions(self):
        j = np.arange(self.nat)
        ix, iy, iz = j % self.nx, (j // self.nx) % self.ny, j // (self.nx * self.ny)
        return np.stack([ix + 1 + self.x0[0], iy + 1 + self.x0[1], iz + 1 + self.x0[2]], axis=1)

    def rhs(self, r):
        """Full complex64 b (3*NAT) for right-hand side r, zero on vacuum sites."""
        inc = self.incid[r]
        ph = np.exp(1j * (self.positions() @ inc.k))
        b = (inc.e[:, None] * ph[None, :]) * (self.iocc != 0)[None, :]
        return b.reshape(-1).astype(np.complex64)

    def adia(self, r, m=None):
        """Full CXADIA (3*NAT) for right-hand side r: 1/alpha of the problem's
        prescription per component, the same on every site (homogeneous)."""
        inc = self.incid[r]
        khat = inc.k / np.linalg.norm(inc.k)
        eps = complex(self.m if m is None else m) ** 2
        ia = inv_alpha_eps(eps, self.kd, khat, inc.e, self.cmdpol)
        return np.repeat(ia.astype(np.complex64), self.nat)

    def aoff(self):
        return np.zeros(3 * self.nat, dtype=np.complex64)


def fft_friendly(n):
    """Smallest m >= n of the form 2^a 3^b 5^c: DDSCAT extends each grid
    dimension this way so that the padded FFT lengths 2m factor into small
    radices; the extra planes are vacuum."""
    m = max(1, int(n))
    while True:
        k = m
        for f in (2, 3, 5):
            while k % f == 0:
                k //= f
        if k == 1:
            return m
        m += 1


FAST_SIDES = (8, 12, 16, 24, 32, 48, 64, 96, 128, 256)


def fast_side(n):
    """Smallest grid side >= n whose padded FFT length 2*side runs on the
    x-first register pipeline (2^k and 3*2^k lengths); falls back to
    fft_friendly above 256."""
    for s in FAST_SIDES:
        if s >= n:
            return s
    return fft_friendly(n)


def embed_ellipsoid(sides, semi, grid="fast"):
    """(grid dims, IOCC) of an ellipsoid filling a box of the given lattice
    sides, placed in a grid extended with vacuum: grid='fast' picks the sides
    of the fast MATVEC path (fast_side), grid='friendly' DDSCAT's 2^a 3^b 5^c
    sizes (fft_friendly), grid='exact' keeps the sides themselves."""
    sx, sy, sz = (int(v) for v in sides)
    ext = {"fast": fast_side, "friendly": fft_friendly, "exact": (lambda v: v)}[grid]
    gx, gy, gz = ext(sx), ext(sy), ext(sz)
    box = ellipsoid_occupancy(sx, sy, sz, semi).reshape(sz, sy, sx)
    occ = np.zeros((gz, gy, gx), dtype=np.int16)
    occ[:sz, :sy, :sx] = box
    return (gx, gy, gz), occ.reshape(-1)


def scattering_planes(k, e01, step_deg=1.0, phis_deg=(0.0, 90.0)):
    """Scattering directions theta = 0..180 deg (step_deg) in the planes
    phi = phis_deg, phi measured from the incident polarisation e01 about k,
    with DDSCAT's SCAT basis: AKS = |k| n, EM1 = theta-hat, EM2 = n x EM1.
    Returns float64 arrays (ndir, 3) aks, em1, em2."""
    k = np.asarray(k, dtype=np.float64)
    kk = float(np.linalg.norm(k))
    kh = k / kk
    e1 = np.real(np.asarray(e01)).astype(np.float64)
    e1 = e1 - kh * float(kh @ e1)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(kh, e1)
    aks, em1, em2 = [], [], []
    for phi in np.deg2rad(np.asarray(phis_deg, dtype=np.float64)):
        u = math.cos(phi) * e1 + math.sin(phi) * e2
        for t in np.deg2rad(np.arange(0.0, 180.0 + 0.5 * step_deg, step_deg)):
            n = math.cos(t) * kh + math.sin(t) * u
            th = -math.sin(t) * kh + math.cos(t) * u
            aks.append(kk * n)
            em1.append(th)
            em2.append(np.cross(n, th))
    return np.array(aks), np.array(em1), np.array(em2)


def make_problem(nx, ny=None, nz=None, m=1.5 + 0.01j, x=5.0, semi=None, orientations=None, iocc=None,
                 cmdpol="GKDLDR"):
    """Ellipsoid (sphere by default) of size parameter x = k*aeff; one RHS per
    (orientation, polarisation) with k along x before rotation and
    polarisations y and z; polarisability prescription cmdpol."""
    _shape_factor((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), cmdpol)  # validates the name
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    if iocc is None:
        iocc = ellipsoid_occupancy(nx, ny, nz, semi)
    nat0 = int(np.count_nonzero(iocc))
    aeff = (3.0 * nat0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    kd = x / aeff
    x0 = (-(nx + 1) / 2.0, -(ny + 1) / 2.0, -(nz + 1) / 2.0)
    p = Problem(nx, ny, nz, np.asarray(iocc, dtype=np.int16), complex(m), kd, aeff, x0, cmdpol=cmdpol)
    if orientations is None:
        orientations = [(0.0, 0.0, 0.0)]
    for ang in orientations:
        R = euler_rotation(*ang)
        k = kd * (R @ np.array([1.0, 0.0, 0.0]))
        for e in (R @ np.array([0.0, 1.0, 0.0]), R @ np.array([0.0, 0.0, 1.0])):
            p.incid.append(Incidence(k=k, e=e.astype(np.complex128)))
    return p


def voxel_problem(n, p_occ=0.6, m1=1.5 + 0.01j, m2=1.2 + 0.0j, x=8.0, seed=0, cmdpol="GKDLDR"):
    """Two-material random voxel target: each voxel occupied with probability
    p_occ, material 1 with probability 1/2.  Returns (Problem, material map)."""
    rng = np.random.default_rng(seed)
    occ = rng.random(n ** 3) < p_occ
    mat = np.where(rng.random(n ** 3) < 0.5, 1, 2) * occ
    prob = make_problem(n, m=m1, x=x, iocc=occ.astype(np.int16), cmdpol=cmdpol)
    return prob, mat
