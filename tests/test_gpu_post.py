"""GPU parity of EVALQ and SCAT (ddscat_cuda_evalq_f32, ddscat_cuda_scat_f32)
against the FP64 oracle evaluated on the same polarisation vector.
Tolerances: 1e-6 relative for EVALQ sums (FP64 reductions of FP32 inputs),
1e-5 for far-field quantities (FP32 phase tables)."""
import math

import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets
from oracle import ddscat_oracle as O


def _solved(n=12, m=1.33 + 0.05j, x=2.0):
    prob = targets.make_problem(n, m=m, x=x)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    out = dda.solve("qmrccg", b, adia, aoff, maxit=500, tol=1e-6)
    occ = prob.occ
    return prob, dda, out, occ, b, adia


@pytest.mark.gpu
def test_evalq_resident_and_compact():
    prob, dda, out, occ, b, adia = _solved()
    k = prob.incid[0].k
    got = dda.evalq(k, use_resident=1)
    pc = O.gather_compact(out.x, occ, prob.nat)
    ec = O.gather_compact(b, occ, prob.nat)
    ac = O.gather_compact(adia, occ, prob.nat)
    rng = np.random.default_rng(1)
    oc = np.zeros_like(ac)
    ref = O.evalq(ec, pc, ac, oc, k, 1.0)
    for g, r in zip(got, ref):
        assert abs(g - r) <= 1e-6 * max(abs(r), 1e-30)
    # compact host inputs with a nonzero off-diagonal block
    oc2 = (0.1 * (rng.normal(size=ac.size) + 1j * rng.normal(size=ac.size))).astype(np.complex64)
    got2 = dda.evalq(k, use_resident=0, e=ec, p=pc, adia=ac, aoff=oc2)
    ref2 = O.evalq(ec, pc, ac, oc2, k, 1.0)
    for g, r in zip(got2, ref2):
        assert abs(g - r) <= 1e-6 * max(abs(r), 1e-30)
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("etasca", [0.5, 3.0])
def test_scat_matches_oracle(etasca):
    prob, dda, out, occ, b, adia = _solved()
    k = prob.incid[0].k
    e01 = prob.incid[0].e
    # selected directions: 0..180 deg in two planes, with the DDSCAT basis vectors
    th = np.deg2rad(np.arange(0, 181, 15.0))
    kk = np.linalg.norm(k)
    aks, em1, em2 = [], [], []
    for phi in (0.0, math.pi / 2):
        for t in th:
            n = np.array([math.cos(t), math.sin(t) * math.cos(phi), math.sin(t) * math.sin(phi)])
            e1 = np.array([-math.sin(t), math.cos(t) * math.cos(phi), math.cos(t) * math.sin(phi)])
            e2 = np.cross(n, e1)
            aks.append(kk * n)
            em1.append(e1)
            em2.append(e2)
    aks, em1, em2 = (np.array(a, dtype=np.float32) for a in (aks, em1, em2))
    got = dda.scat(k, e01, prob.x0, etasca=etasca, aks=aks, em1=em1, em2=em2)
    pc = O.gather_compact(out.x, occ, prob.nat)
    ref = O.scat(pc, occ, prob.nx, prob.ny, 0, k, aks, (1, 1, 1), em1, em2, 1.0, etasca, e01, prob.x0)
    assert got["navg"] == len(O.scat_integration_dirs(k, e01, etasca, occ.size)[0])
    assert abs(got["csca"] - ref["csca"]) <= 1e-5 * ref["csca"]
    assert abs(got["cscag2"] - ref["cscag2"]) <= 1e-5 * ref["cscag2"]
    for a, r in zip(got["cscag"], ref["cscag"]):
        assert abs(a - r) <= 1e-5 * ref["csca"]
    assert abs(got["cbksca"] - ref["cbksca"]) <= 1e-5 * max(ref["cbksca"], 1e-6 * ref["csca"])
    fmax = max(np.abs(ref["f1"]).max(), np.abs(ref["f2"]).max())
    assert np.abs(got["f1"] - ref["f1"]).max() <= 1e-5 * fmax
    assert np.abs(got["f2"] - ref["f2"]).max() <= 1e-5 * fmax
    dda.release()


@pytest.mark.gpu
def test_energy_conservation_on_gpu():
    """Cext = Cabs + Csca from the GPU's own EVALQ and SCAT (fine quadrature)."""
    prob, dda, out, occ, b, adia = _solved(n=16, x=2.5)
    k = prob.incid[0].k
    cabs, cext, _ = dda.evalq(k)
    sc = dda.scat(k, prob.incid[0].e, prob.x0, etasca=0.2)
    assert cext == pytest.approx(cabs + sc["csca"], rel=3e-3)
    dda.release()


def _plane_dirs(kk, phi, th_deg):
    """Scattering directions for incidence along x in the plane at azimuth phi,
    with DDSCAT's basis EM1 = theta-hat, EM2 = n x EM1 (= phi-hat)."""
    aks, em1, em2 = [], [], []
    for t in np.deg2rad(th_deg):
        n = np.array([math.cos(t), math.sin(t) * math.cos(phi), math.sin(t) * math.sin(phi)])
        e1 = np.array([-math.sin(t), math.cos(t) * math.cos(phi), math.cos(t) * math.sin(phi)])
        aks.append(kk * n)
        em1.append(e1)
        em2.append(np.cross(n, e1))
    return (np.array(a, dtype=np.float32) for a in (aks, em1, em2))


@pytest.mark.gpu
def test_mueller_matches_oracle():
    rng = np.random.default_rng(17)
    nd = 200
    k = np.array([0.7, 0.2, -0.3])
    e01 = np.array([0.1 + 0.2j, 0.9, 0.3j])
    e01 /= np.linalg.norm(e01)
    e02 = np.cross(k / np.linalg.norm(k), np.conj(e01))
    em2 = rng.normal(size=(nd, 3)).astype(np.float32)
    f = [(rng.normal(size=nd) + 1j * rng.normal(size=nd)).astype(np.complex64) for _ in range(4)]
    dda = D.DDA()
    s, m = dda.mueller(k, e01, e02, em2, *f)
    sref = O.amplitude_matrix(k.astype(np.float32), e01.astype(np.complex64), e02.astype(np.complex64), em2, *f)
    mref = O.mueller_from_amplitude(sref)
    assert np.abs(s - sref).max() <= 1e-5 * np.abs(sref).max()
    assert np.abs(m - mref).max() <= 1e-5 * np.abs(mref).max()


@pytest.mark.gpu
def test_mueller_of_dda_sphere():
    """S_ij of a solved DDA sphere in its mirror plane (incidence along x,
    scattering plane x-y): S3 = S4 = 0 by symmetry, so the off-block elements
    vanish, S11 = S22, S33 = S44, S12 = S21, S34 = -S43; forward, S33 = S11 and
    S12 = 0; and sum_ij S_ij^2 = 4 S11^2 (a pure Mueller matrix)."""
    n = 16
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=2.5)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    k = prob.incid[0].k
    aks, em1, em2 = _plane_dirs(np.linalg.norm(k), 0.0, np.arange(0, 181, 5.0))
    f = {}
    for l in (0, 1):
        inc = prob.incid[l]
        dda.solve("qmrccg", prob.rhs(l), prob.adia(l), prob.aoff(), maxit=500, tol=1e-6)
        sc = dda.scat(k, inc.e, prob.x0, etasca=3.0, aks=aks, em1=em1, em2=em2)
        f[l] = (sc["f1"], sc["f2"])
    s, m = dda.mueller(k, prob.incid[0].e, prob.incid[1].e, em2, f[0][0], f[0][1], f[1][0], f[1][1])
    s11 = m[:, 0, 0]
    assert np.all(s11 > 0)
    for i, j in [(0, 2), (0, 3), (1, 2), (1, 3), (2, 0), (2, 1), (3, 0), (3, 1)]:
        assert np.abs(m[:, i, j]).max() <= 1e-4 * s11.max(), (i, j)
    assert np.allclose(m[:, 1, 1], s11, rtol=1e-4, atol=1e-6 * s11.max())
    assert np.allclose(m[:, 3, 3], m[:, 2, 2], rtol=1e-4, atol=1e-6 * s11.max())
    assert np.allclose(m[:, 0, 1], m[:, 1, 0], atol=1e-6 * s11.max())
    assert np.allclose(m[:, 2, 3], -m[:, 3, 2], atol=1e-6 * s11.max())
    assert abs(m[0, 2, 2] - s11[0]) <= 1e-4 * s11[0] and abs(m[0, 0, 1]) <= 1e-4 * s11[0]
    assert np.allclose(np.sum(m ** 2, axis=(1, 2)), 4 * s11 ** 2, rtol=1e-5)
    dda.release()


@pytest.mark.gpu
def test_scat_amplitudes_f64_matches_oracle_and_fp32_scat():
    """ddscat_b200_scat_amplitudes_f64 equals the FP64 oracle far-field sums
    (1e-11 relative) and the FP32 SCAT amplitudes of the same polarisation to
    the FP32 phase-table tolerance (1e-5 of the largest amplitude)."""
    prob, dda, out, occ, b, adia = _solved()
    k = prob.incid[0].k
    e01 = prob.incid[0].e
    aks, em1, em2 = targets.scattering_planes(k, e01, step_deg=5.0)
    x64 = out.x.astype(np.complex128)[None, :]
    f1, f2 = dda.scat_amplitudes_f64(x64, k, aks, em1, em2, prob.x0)
    pc = O.gather_compact(x64[0], occ, prob.nat)
    sums = O.farfield_sums(pc, occ, prob.nx, prob.ny, aks, (1.0, 1.0, 1.0), prob.x0)
    term = np.linalg.norm(k) ** 3
    r1 = term * np.einsum("dc,dc->d", em1, sums)
    r2 = term * np.einsum("dc,dc->d", em2, sums)
    scale = max(np.abs(r1).max(), np.abs(r2).max())
    assert np.abs(f1[0] - r1).max() <= 1e-11 * scale
    assert np.abs(f2[0] - r2).max() <= 1e-11 * scale
    sc = dda.scat(k, e01, prob.x0, etasca=0.5, aks=aks.astype(np.float32), em1=em1.astype(np.float32),
                  em2=em2.astype(np.float32))
    assert np.abs(sc["f1"] - f1[0]).max() <= 1e-5 * scale
    assert np.abs(sc["f2"] - f2[0]).max() <= 1e-5 * scale
    dda.release()


@pytest.mark.gpu
def test_mueller_f64_matches_oracle_and_f32():
    """ddscat_b200_mueller_f64 equals the oracle's Bohren & Huffman amplitude and
    Mueller matrices to 1e-12 and agrees with the complex-float entry point on
    the same (rounded) amplitudes to 1e-6 of S11."""
    rng = np.random.default_rng(4)
    k = np.array([0.3, -0.2, 0.5])
    e01, e02 = np.array([0.0, 1.0, 0.0], dtype=np.complex128), np.array([0.0, 0.0, 1.0], dtype=np.complex128)
    aks, em1, em2 = targets.scattering_planes(k, np.cross(k, [1.0, 0.0, 0.0]), step_deg=10.0)
    nd = aks.shape[0]
    f = [rng.normal(size=nd) + 1j * rng.normal(size=nd) for _ in range(4)]
    dda = D.DDA()
    s64, m64 = dda.mueller_f64(k, e01, e02, em2, *f)
    S = O.amplitude_matrix(k, e01, e02, em2, *f)
    M = O.mueller_from_amplitude(S)
    assert np.abs(s64 - S).max() <= 1e-12 * np.abs(S).max()
    assert np.abs(m64 - M).max() <= 1e-12 * np.abs(M).max()
    s32, m32 = dda.mueller(k.astype(np.float32), e01, e02, em2.astype(np.float32), *[v.astype(np.complex64) for v in f])
    assert np.abs(m32 - m64).max() <= 1e-6 * np.abs(m64[:, 0, 0]).max()


@pytest.mark.gpu
def test_scat_csca_f64_matches_oracle_and_fp32_scat():
    """ddscat_b200_scat_csca_f64 gives the oracle's SCAT cross sections (same
    directions and weights, FP64 sums) to 1e-10 relative, two RHS per call,
    and agrees with the FP32 SCAT of the same polarisation to the FP32
    phase-table tolerance (1e-5 relative for Csca, 1e-5 absolute for g)."""
    prob, dda, out, occ, b, adia = _solved()
    k = prob.incid[0].k
    e01 = prob.incid[0].e
    x64 = np.stack([out.x.astype(np.complex128), 0.5j * out.x.astype(np.complex128)])
    e01s = np.stack([e01, e01])
    got = dda.scat_csca_f64(x64, k, e01s, prob.x0, etasca=0.5)
    pc = O.gather_compact(x64[0], occ, prob.nat)
    ref = O.scat(pc, occ, prob.nx, prob.ny, 0, k, np.zeros((0, 3)), (1.0, 1.0, 1.0), None, None, 1.0, 0.5, e01,
                 prob.x0)
    assert got["navg"][0] == ref["navg"] == got["navg"][1]
    assert abs(got["csca"][0] - ref["csca"]) <= 1e-10 * ref["csca"]
    assert np.abs(got["cscag"][0] - np.array(ref["cscag"])).max() <= 1e-10 * ref["csca"]
    assert abs(got["cscag2"][0] - ref["cscag2"]) <= 1e-10 * ref["csca"]
    assert abs(got["cbksca"][0] - ref["cbksca"]) <= 1e-10 * ref["csca"]
    # the second RHS is 0.5i times the first: |0.5|^2 of every cross section
    assert abs(got["csca"][1] - 0.25 * got["csca"][0]) <= 1e-12 * got["csca"][0]
    dda.evalq(k, use_resident=1)
    sc = dda.scat(k, e01, prob.x0, etasca=0.5)
    assert sc["navg"] == got["navg"][0]
    assert abs(sc["csca"] - got["csca"][0]) <= 1e-5 * got["csca"][0]
    assert abs(sc["cscag"][0] / sc["csca"] - got["cscag"][0, 0] / got["csca"][0]) <= 1e-5
    dda.release()
