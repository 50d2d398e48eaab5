"""Seeded inputs of the edge cases that tests/golden/make_reference_fixtures.py
runs through the reference library (reference_fixtures_edge.npz) and that
tests/test_gpu_edge.py runs through this library (test inputs only)."""
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
