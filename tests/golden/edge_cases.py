"""Seeded inputs of the edge cases and periodic targets that
tests/golden/make_reference_fixtures.py runs through the reference library
(reference_fixtures_edge.npz, reference_fixtures_pbc.npz) and that the tests
run through the oracle and this library (test inputs only)."""
import numpy as np

from ddscat_b200 import targets

SOLVERS_AOFF = ("pbcgs2", "qmrccg", "pbcgst", "petrkp", "gpbicg")
HOLLOW = ("hollow16", "hollow18x12x10")
TOL, MAXIT = 1e-5, 600


def aoff_problem():
    """10x9x8 ellipsoid with anisotropic sites: nonzero CXAOFF, symmetric per
    site (the matrix stays complex symmetric), zero on vacuum sites."""
    prob = targets.make_problem(10, 9, 8, m=1.5 + 0.02j, x=1.5)
    rng = np.random.default_rng(11)
    b, adia = prob.rhs(0), prob.adia(0)
    aoff = (0.4 * (rng.normal(size=b.size) + 1j * rng.normal(size=b.size))).astype(np.complex64)
    aoff.reshape(3, -1)[:, prob.iocc == 0] = 0
    return prob, b, adia, aoff


def _hollow(n):
    c = (np.arange(n) + 0.5 - n / 2) / (n / 2)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    r2 = x * x + y * y + z * z
    shell = (r2 <= 1.0) & (r2 >= 0.6)
    blob1 = (x - 0.1) ** 2 + (y + 0.05) ** 2 + z ** 2 <= 0.04
    blob2 = (x + 0.05) ** 2 + (y - 0.1) ** 2 + (z - 0.05) ** 2 <= 0.01
    occ = shell | blob1 | blob2
    occ[:, :, n // 2] = False  # a vacant yz plane
    occ[n // 3, :, :] = False  # a vacant xy plane
    return occ.astype(np.int16)


def sparse_problem(case):
    """single_site: one occupied site of a 4^3 grid; hollow16 / hollow18x12x10:
    a shell with two separated blobs and vacant planes (rows, columns and
    planes partly or wholly vacant).  Returns (prob, b, adia, aoff, x) with a
    seeded MATVEC input x."""
    if case == "single_site":
        dims = (4, 4, 4)
        iocc = np.zeros(64, dtype=np.int16)
        iocc[1 + 4 * (2 + 4 * 3)] = 1
    elif case == "hollow16":
        dims = (16, 16, 16)
        iocc = _hollow(16).reshape(-1)
    else:
        dims = (18, 12, 10)
        iocc = np.ascontiguousarray(_hollow(18)[:10, :12, :18]).reshape(-1)
    prob = targets.make_problem(*dims, m=1.6 + 0.05j, x=1.0, iocc=iocc)
    rng = np.random.default_rng(5)
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    x = (rng.normal(size=b.size) + 1j * rng.normal(size=b.size)).astype(np.complex64)
    return prob, b, adia, aoff, x


def pbc_cases():
    """Periodic MATVEC cases (name, dims, idipint, gamma, pyd, pzd, ak) and the
    seeded inputs of each (80 % occupancy, random x zero on vacuum sites,
    CXADIA shifted by 4 for a well-conditioned operator, CXAOFF); PYD and PZD are the periods in lattice units (dx = 1)."""
    cases = [("y", (4, 3, 3), 0, 5e-2, 3.0, 0.0, (0.6, 0.25, 0.0)),
             ("z", (6, 4, 4), 0, 5e-2, 0.0, 4.0, (0.5, 0.0, 0.3)),
             ("yz", (6, 4, 4), 0, 5e-2, 4.0, 4.0, (0.6, 0.1, 0.05)),
             ("yf", (5, 4, 4), 1, 5e-2, 4.0, 0.0, (0.55, 0.2, 0.1))]
    out = []
    rng = np.random.default_rng(4242)
    for name, dims, idip, gamma, pyd, pzd, ak in cases:
        nat = int(np.prod(dims))
        iocc = (rng.random(nat) < 0.8).astype(np.int16)
        iocc[0] = 1
        c = lambda s=1.0: (s * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)  # noqa: E731
        x, adia, aoff = c(), c(), c(0.3)
        adia += np.complex64(4.0)
        x[np.tile(iocc == 0, 3)] = 0
        out.append(dict(name=name, dims=dims, idipint=idip, gamma=gamma, pyd=pyd, pzd=pzd,
                        ak=np.array(ak, dtype=np.float32), iocc=iocc, x=x, adia=adia, aoff=aoff))
    return out


def pbc_solve_problem():
    """A slab periodic in y and z: a 6 x 4 x 4 cell fully occupied, GKDLDR
    CXADIA of m = 1.5+0.01i (targets.make_problem), incident along x
    (k_perp = |k_x|), PBCGS2 at tol 1e-5; SCAT amplitudes in three directions.
    Returns (prob, gamma, pyd, pzd, aks, em1, em2)."""
    prob = targets.make_problem(6, 4, 4, m=1.5 + 0.01j, x=1.5, iocc=np.ones(96, dtype=np.int16))
    th = np.deg2rad([0.0, 60.0, 180.0])
    kk = float(np.linalg.norm(prob.incid[0].k))
    aks = np.array([[kk * np.cos(t), kk * np.sin(t), 0.0] for t in th], dtype=np.float32)
    em1 = np.array([[-np.sin(t), np.cos(t), 0.0] for t in th], dtype=np.float32)
    em2 = np.array([[0.0, 0.0, 1.0] for t in th], dtype=np.float32)
    return prob, 5e-2, 4.0, 4.0, aks, em1, em2


def pbc_cpu_green_case():
    """prepare_f32 with IPBC = 1: a caller-supplied full-grid spectrum of the
    six tensor components, planar (6, 2nz, 2ny, 2nx) complex64 (random, seeded:
    the MATVEC's full-tensor branch and the spectrum's layout do not depend on
    its values being a Green tensor), on a 6 x 5 x 4 grid with random inputs."""
    rng = np.random.default_rng(777)
    dims = (6, 5, 4)
    nat = int(np.prod(dims))
    shape = (6, 2 * dims[2], 2 * dims[1], 2 * dims[0])
    green = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    iocc = (rng.random(nat) < 0.8).astype(np.int16)
    iocc[0] = 1
    c = lambda s=1.0: (s * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)  # noqa: E731
    x, adia, aoff = c(), c(), c(0.3)
    x[np.tile(iocc == 0, 3)] = 0
    return dict(dims=dims, green=green, iocc=iocc, x=x, adia=adia, aoff=aoff)


DX = (1.0, 0.9, 1.1)


def dx_cases():
    """Rectangular lattices, DX = (1.0, 0.9, 1.1) (prepare_green's dx1..dx3):
    MATVEC cases (name, dims, ipbc, idipint, gamma, pyd, ak) with seeded inputs
    as in pbc_cases; the periodic one exercises the period PYD * DX(2) and the
    replica offsets jpy * PYD * DX(2) * DX(2) of cu:642 and cu:1012."""
    cases = [("iso", (7, 6, 5), 0, 0, 0.0, 0.0, (0.35, -0.2, 0.3)),
             ("flt", (7, 6, 5), 0, 1, 0.0, 0.0, (0.35, -0.2, 0.3)),
             ("pbc", (5, 4, 4), 1, 0, 5e-2, 4.0, (0.55, 0.2, 0.1))]
    out = []
    rng = np.random.default_rng(99)
    for name, dims, ipbc, idip, gamma, pyd, ak in cases:
        nat = int(np.prod(dims))
        iocc = (rng.random(nat) < 0.8).astype(np.int16)
        iocc[0] = 1
        c = lambda s=1.0: (s * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)  # noqa: E731
        x, adia, aoff = c(), c(), c(0.3)
        adia += np.complex64(4.0)
        x[np.tile(iocc == 0, 3)] = 0
        out.append(dict(name=name, dims=dims, ipbc=ipbc, idipint=idip, gamma=gamma, pyd=pyd,
                        ak=np.array(ak, dtype=np.float32), iocc=iocc, x=x, adia=adia, aoff=aoff))
    return out


def dx_solve_problem():
    """A 10 x 8 x 6 ellipsoid on the DX lattice (m = 1.5+0.01i, x = 2), QMRCCG at
    tol 1e-5, EVALQ, and SCAT at ETASCA 3.0 (site positions ((i+1)+x0)*DX) with
    amplitudes in seven directions of the xy plane."""
    prob = targets.make_problem(10, 8, 6, m=1.5 + 0.01j, x=2.0)
    th = np.deg2rad(np.arange(0.0, 181.0, 30.0))
    kk = float(np.linalg.norm(prob.incid[0].k))
    aks = np.array([[kk * np.cos(t), kk * np.sin(t), 0.0] for t in th], dtype=np.float32)
    em1 = np.array([[-np.sin(t), np.cos(t), 0.0] for t in th], dtype=np.float32)
    em2 = np.array([[0.0, 0.0, 1.0] for t in th], dtype=np.float32)
    return prob, aks, em1, em2


def limits_problem():
    """The solvers' limit cases on a 12^3 sphere (m = 1.5+0.01i, x = 2): MAXIT
    reached (maxit 3 at tol 1e-12), a zero right-hand side (maxit 10), and a
    nonzero initial guess (seeded, zero on vacuum sites; maxit 300, tol 1e-5).
    Returns (prob, b, adia, aoff, x0)."""
    prob = targets.make_problem(12, m=1.5 + 0.01j, x=2.0)
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    rng = np.random.default_rng(314)
    x0 = (0.05 * (rng.normal(size=b.size) + 1j * rng.normal(size=b.size))).astype(np.complex64)
    x0.reshape(3, -1)[:, prob.iocc == 0] = 0
    return prob, b, adia, aoff, x0
