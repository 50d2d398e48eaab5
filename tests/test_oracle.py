"""CPU tests of the oracle itself: it is checked against an independent dense
assembly of the operator, the reference's own numeric scripts (restated), and
physical identities, before it is trusted as the checker for the CUDA path."""
import math

import numpy as np
import pytest

from oracle import ddscat_oracle as O
from ddscat_b200 import targets


def _rand_c(rng, n):
    return (rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex128)


# -- ddscat_cuda_unified/scripts/check_compact_mapping.py (restated) --------
def test_compact_mapping_roundtrip():
    nat = 10
    iocc = np.zeros(nat, dtype=np.int16)
    iocc[[0, 2, 5, 9]] = 1
    occ = O.occupied_index(iocc)
    assert list(occ) == [0, 2, 5, 9]
    full = (np.arange(3 * nat) + 1j * np.arange(3 * nat) / 10).astype(np.complex64)
    comp = O.gather_compact(full, occ, nat)
    assert comp.size == 3 * occ.size
    for q in range(3 * occ.size):
        c, k = divmod(q, occ.size)
        assert comp[q] == full[c * nat + occ[k]]
    back = O.scatter_full(comp, occ, nat)
    expected = np.zeros_like(full)
    for c in range(3):
        expected[c * nat + occ] = full[c * nat + occ]
    assert np.array_equal(back, expected)


# -- ddscat_cuda_unified/scripts/test_gpu_final_sections_math.py (restated) --
def test_final_sections_identities():
    rng = np.random.default_rng(12345)
    N = 257
    r = rng.normal(size=(N, 3))
    p = rng.normal(size=(N, 3)) + 1j * rng.normal(size=(N, 3))
    k = rng.normal(size=3)
    k *= 2.3 / np.linalg.norm(k)
    n = k / np.linalg.norm(k)
    phase = np.exp(-1j * (r @ k))
    orig = np.sum((p - n[None, :] * np.sum(p * n[None, :], axis=1)[:, None]) * phase[:, None], axis=0)
    s = np.sum(p * phase[:, None], axis=0)
    assert np.allclose(orig, s - n * np.dot(n, s), rtol=2e-13, atol=2e-13)
    em = rng.normal(size=3)
    em -= n * np.dot(n, em)
    em /= np.linalg.norm(em)
    assert np.allclose(np.sum((p @ em) * phase), np.dot(em, s), rtol=2e-13, atol=2e-13)
    ad = rng.normal(size=(N, 3)) + 1j * rng.normal(size=(N, 3))
    ao = rng.normal(size=(N, 3)) + 1j * rng.normal(size=(N, 3))
    k3 = 1.7
    # the oracle's EVALQ q-vector against the block form
    pc = p.T.reshape(-1)
    adc = ad.T.reshape(-1)
    aoc = ao.T.reshape(-1)
    akv = (k3 ** (1.0 / 3.0), 0.0, 0.0)
    cabs, cext, cpha = O.evalq(pc, pc, adc, aoc, akv, 1.0)
    q = np.empty_like(p)
    q[:, 0] = (ad[:, 0] + 1j * k3 / 1.5) * p[:, 0] + ao[:, 1] * p[:, 2] + ao[:, 2] * p[:, 1]
    q[:, 1] = (ad[:, 1] + 1j * k3 / 1.5) * p[:, 1] + ao[:, 2] * p[:, 0] + ao[:, 0] * p[:, 2]
    q[:, 2] = (ad[:, 2] + 1j * k3 / 1.5) * p[:, 2] + ao[:, 0] * p[:, 1] + ao[:, 1] * p[:, 0]
    z2 = sum(np.vdot(p[j], q[j]) for j in range(N))
    akk = k3 ** (1.0 / 3.0)
    assert cabs == pytest.approx(-4 * math.pi * akk * z2.imag, rel=1e-12)
    # far-field sums: projection after summing equals summing projections
    occ = np.arange(N)
    sums = O.farfield_sums(pc, occ, N, 1, [k], (1, 1, 1), (0, 0, 0))
    rr = np.stack([occ + 1.0, np.ones(N), np.ones(N)], axis=1)
    direct = np.sum(p * np.exp(-1j * (rr @ k))[:, None], axis=0)
    assert np.allclose(sums[0], direct, rtol=1e-12)


@pytest.mark.parametrize("dims", [(4, 4, 4), (5, 3, 4), (6, 6, 6)])
@pytest.mark.parametrize("idipint", [0, 1])
@pytest.mark.parametrize("cwhat", ["N", "C"])
def test_fft_matvec_equals_dense(dims, idipint, cwhat):
    """The FFT operator (octant Green, sign rules, pad/trim) equals a dense
    O(N^2) assembly of A (independent of any FFT)."""
    nx, ny, nz = dims
    rng = np.random.default_rng(7)
    nat = nx * ny * nz
    iocc = (rng.random(nat) < 0.8).astype(np.int16)
    ak = (0.7, 0.2, -0.1)
    gp = O.GreenParams(nx, ny, nz, idipint=idipint, ak=ak)
    op = O.Operator.from_octant(nx, ny, nz, O.green_octant(gp), iocc)
    x = _rand_c(rng, 3 * nat)
    adia = _rand_c(rng, 3 * nat)
    aoff = _rand_c(rng, 3 * nat)
    y = op.apply_full(x, adia, aoff, cwhat)
    A = O.dense_matrix(nx, ny, nz, iocc, adia, aoff, gp.akd, idipint)
    yd = A @ x if cwhat == "N" else np.conj(A) @ x
    assert np.allclose(y, yd, rtol=1e-10, atol=1e-10 * np.abs(yd).max())


def test_operator_is_complex_symmetric():
    nx = ny = nz = 4
    rng = np.random.default_rng(3)
    nat = nx * ny * nz
    iocc = np.ones(nat, dtype=np.int16)
    adia = _rand_c(rng, 3 * nat)
    aoff = _rand_c(rng, 3 * nat)
    A = O.dense_matrix(nx, ny, nz, iocc, adia, aoff, 0.9, 0)
    assert np.allclose(A, A.T, atol=1e-12)


def test_octant_expansion_matches_full_spectrum():
    gp = O.GreenParams(5, 4, 3, ak=(0.5, 0.3, 0.2))
    full = O.green_spectrum_full(gp)
    rebuilt = O.expand_octant(O.green_octant(gp), 5, 4, 3)
    assert np.allclose(full, rebuilt, atol=1e-11 * np.abs(full).max())


def test_scat_quadrature_weights():
    dirs, w = O.scat_integration_dirs((0.8, 0.0, 0.0), (0, 1, 0), 0.5, 1000)
    assert w[:, 0].sum() == pytest.approx(4 * math.pi, rel=1e-12)
    # directions have |k_s| = |k|
    assert np.allclose(np.linalg.norm(dirs.astype(np.float64), axis=1), 0.8, rtol=1e-6)
    assert np.allclose(dirs[-1], (-0.8, 0, 0), atol=1e-6)  # last direction is backscatter


def _small_problem(n=8, m=1.5 + 0.01j, x=1.5):
    prob = targets.make_problem(n, m=m, x=x)
    gp = O.GreenParams(n, n, n, ak=tuple(prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    occ = op.occ
    b = O.gather_compact(prob.rhs(0), occ, prob.nat)
    adia = O.gather_compact(prob.adia(0), occ, prob.nat)
    aoff = np.zeros_like(adia)
    mv = lambda v: op.apply_compact(v, adia, aoff)  # noqa: E731
    mvh = lambda v: op.apply_compact(v, adia, aoff, "C")  # noqa: E731
    return prob, op, b, adia, aoff, mv, mvh


@pytest.mark.parametrize("name", ["pbcgs2", "qmrccg", "gpbicg", "bicgstab4", "gpbicgstab2", "gpbicgstab4", "pbcgst",
                                  "petrkp"])
def test_oracle_solvers_converge(name):
    prob, op, b, adia, aoff, mv, mvh = _small_problem()
    x0 = np.zeros_like(b)
    tol = 1e-6
    if name == "pbcgst":
        res = O.solve_pbcgst(mv, b, x0, 300, tol, adia)
    elif name == "petrkp":
        res = O.solve_petrkp(mv, mvh, b, x0, 300, tol)
    else:
        res = O.SOLVERS[name](mv, b, x0, 300, tol)
    assert res.status == 0
    true = np.linalg.norm(b - mv(res.x)) / np.linalg.norm(b)
    assert true <= 1.01 * tol
    assert res.tole <= tol * 1.01
    # same solution as a dense direct solve
    A = np.stack([mv(np.eye(b.size)[:, i]) for i in range(b.size)], axis=1)
    xd = np.linalg.solve(A, b)
    assert np.linalg.norm(res.x - xd) / np.linalg.norm(xd) < 1e-4


def test_optical_theorem():
    """Cext = Cabs + Csca for a converged solve (energy conservation)."""
    prob, op, b, adia, aoff, mv, mvh = _small_problem(n=8, m=1.33 + 0.05j, x=1.0)
    res = O.solve_qmrccg(mv, b, np.zeros_like(b), 500, 1e-8)
    ak = prob.incid[0].k
    cabs, cext, _ = O.evalq(b, res.x, adia, aoff, ak, 1.0)
    sc = O.scat(res.x, op.occ, prob.nx, prob.ny, 0, ak, [], (1, 1, 1), [], [], 1.0, 0.2, prob.incid[0].e, prob.x0)
    assert cext == pytest.approx(cabs + sc["csca"], rel=2e-3)


def test_mueller_identities():
    """Bohren & Huffman eq. 3.16 from a single amplitude matrix: the Mueller
    matrix is 'pure', so sum_ij S_ij^2 = 4 S_11^2; with S3 = S4 = 0 (sphere)
    the off-block elements vanish, S11 = S22, S33 = S44, S12 = S21, S34 = -S43."""
    rng = np.random.default_rng(3)
    S = rng.normal(size=(50, 4)) + 1j * rng.normal(size=(50, 4))
    M = O.mueller_from_amplitude(S)
    assert np.allclose(np.sum(M ** 2, axis=(1, 2)), 4 * M[:, 0, 0] ** 2, rtol=1e-12)
    S[:, 2:] = 0
    M = O.mueller_from_amplitude(S)
    for i, j in [(0, 2), (0, 3), (1, 2), (1, 3), (2, 0), (2, 1), (3, 0), (3, 1)]:
        assert np.allclose(M[:, i, j], 0)
    assert np.allclose(M[:, 0, 0], M[:, 1, 1]) and np.allclose(M[:, 2, 2], M[:, 3, 3])
    assert np.allclose(M[:, 0, 1], M[:, 1, 0]) and np.allclose(M[:, 2, 3], -M[:, 3, 2])


def test_amplitude_matrix_forward_direction():
    """Forward scattering by an isotropic scatterer keeps the incident
    polarisation, f_ml = f0 (e_m . e0l), so S1 = S2 = -i f0 and S3 = S4 = 0
    for any azimuth of the scattering plane (DDSCAT basis EM2 = n x EM1)."""
    k = np.array([2.0, 0.0, 0.0])
    e01 = np.array([0, 1, 0], dtype=complex)
    e02 = np.array([0, 0, 1], dtype=complex)
    f0 = 0.3 - 0.7j
    for phi in np.linspace(0, np.pi, 5):
        em1 = np.array([0.0, np.cos(phi), np.sin(phi)])  # theta-hat at theta = 0
        em2 = np.cross(k / 2, em1)
        f = [[f0 * np.dot(em, e) for e in (e01, e02)] for em in (em1, em2)]
        S = O.amplitude_matrix(k, e01, e02, em2[None, :], [f[0][0]], [f[1][0]], [f[0][1]], [f[1][1]])
        assert np.allclose(S[0, 0], S[0, 1]) and np.allclose(S[0, 2:], 0)
        assert np.allclose(S[0, 0], -1j * f0)
