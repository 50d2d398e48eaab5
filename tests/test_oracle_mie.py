"""Physics checks of the oracle against the Mie series of a homogeneous sphere
(CPU).  The Mie code (oracle/mie.py) is first checked against the Rayleigh
limit and the optical theorem; the oracle's FP64 DDA of a lattice sphere (LDR
or GKDLDR polarisability, volume-equivalent radius from NAT0) must then reproduce Mie's
Q_ext and Q_abs, and the Mueller matrix elements of its far field (SCAT f_ml,
amplitude matrix S = -i f, Bohren & Huffman eq. 3.16), within the DDA
discretisation error, which is about 1 % at |m| k d < 0.5."""
import math

import numpy as np
import pytest

from ddscat_b200 import targets
from oracle import ddscat_oracle as O
from oracle.mie import mie_amplitudes, mie_efficiencies


@pytest.mark.parametrize("x,m", [(0.02, 1.5 + 0.1j), (0.05, 1.33 + 0.01j)])
def test_mie_rayleigh_limit(x, m):
    """Q_abs -> 4x Im(alpha), Q_sca -> 8/3 x^4 |alpha|^2, alpha = (m^2-1)/(m^2+2),
    with relative corrections of order x^2."""
    qext, qsca, qabs, g = mie_efficiencies(x, m)
    al = (m * m - 1) / (m * m + 2)
    assert qabs == pytest.approx(4 * x * al.imag, rel=2e-3)
    assert qsca == pytest.approx(8.0 / 3.0 * x ** 4 * abs(al) ** 2, rel=2e-3)
    assert abs(g) < 1e-3


def test_mie_real_index_does_not_absorb():
    qext, qsca, qabs, g = mie_efficiencies(5.0, 1.5 + 0.0j)
    assert abs(qabs) < 1e-10 * qext
    assert 0.0 < g < 1.0


@pytest.mark.parametrize("n,m,x,cmdpol,tol_ext,tol_abs,tol_pha,tol_bk", [
    (16, 1.33 + 0.1j, 1.0, "LATTDR", 0.01, 0.01, 0.01, 0.02),
    (16, 1.33 + 0.1j, 1.0, "GKDLDR", 0.01, 0.01, 0.01, 0.02),
    # the small plain-path configuration: 32^3 sphere, m = 1.50 + 0.01i, x = 5
    # (the backscatter of a lattice sphere carries the largest DDA error; with
    # GKDLDR Q_ext and Q_abs are within 0.2 % and 0.3 % of Mie, Q_pha 3.4 % and
    # the backscatter 20 %, with LDR 0.3 %, 1.5 %, 2.1 % and 9 %)
    (32, 1.5 + 0.01j, 5.0, "LATTDR", 0.01, 0.03, 0.03, 0.15),
    (32, 1.5 + 0.01j, 5.0, "GKDLDR", 0.005, 0.01, 0.04, 0.25),
])
def test_oracle_dda_sphere_matches_mie(n, m, x, cmdpol, tol_ext, tol_abs, tol_pha, tol_bk):
    """Q_ext, Q_abs, Q_pha (EVALQ) and Q_sca, g, the backscatter (SCAT's
    angular integration at ETASCA = 0.5, whose last direction is -k) of the
    lattice sphere, averaged over both polarisations.  Q_pha is DDSCAT's
    phase-lag efficiency, -2/x^2 Im S(0) in Bohren & Huffman's convention
    (positive for a small sphere with Re m > 1); CBKSCA is the differential
    cross section at 180 deg, |S1(pi)|^2 / k^2."""
    prob = targets.make_problem(n, m=m, x=x, cmdpol=cmdpol)
    gp = O.GreenParams(n, n, n, ak=tuple(prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    k = prob.incid[0].k
    khat = np.asarray(k) / np.linalg.norm(k)
    area = math.pi * prob.aeff ** 2
    qext, qabs, qpha, qsca, g, qbk = [], [], [], [], [], []
    for r in range(2):  # both incident polarisations
        b = O.gather_compact(prob.rhs(r), op.occ, prob.nat)
        adia = O.gather_compact(prob.adia(r), op.occ, prob.nat)
        aoff = np.zeros_like(adia)
        res = O.solve_qmrccg(lambda v: op.apply_compact(v, adia, aoff), b, np.zeros_like(b), 1000, 1e-6)
        assert res.status == 0
        cabs, cext, cpha = O.evalq(b, res.x, adia, aoff, k, 1.0)
        sc = O.scat(res.x, op.occ, prob.nx, prob.ny, 0, k, [], (1, 1, 1), [], [], 1.0, 0.5, prob.incid[r].e, prob.x0)
        qext.append(cext / area)
        qabs.append(cabs / area)
        qpha.append(cpha / area)
        qsca.append(sc["csca"] / area)
        qbk.append(sc["cbksca"] / area)
        g.append(float(np.dot(sc["cscag"], khat)) / sc["csca"])
    me, ms, ma, mg = mie_efficiencies(x, m)
    s1, _ = mie_amplitudes(x, m, np.array([0.0, math.pi]))
    assert np.mean(qpha) == pytest.approx(-2.0 / x ** 2 * s1[0].imag, rel=tol_pha)
    assert np.mean(qbk) == pytest.approx(abs(s1[1]) ** 2 / (math.pi * x ** 2), rel=tol_bk)
    assert np.mean(qext) == pytest.approx(me, rel=tol_ext)
    assert np.mean(qabs) == pytest.approx(ma, rel=tol_abs)
    assert np.mean(qsca) == pytest.approx(ms, rel=0.02)
    assert abs(np.mean(g) - mg) < 0.01


def test_mie_forward_amplitude_optical_theorem():
    x, m = 2.0, 1.5 + 0.05j
    s1, s2 = mie_amplitudes(x, m, np.array([0.0]))
    assert s1[0] == pytest.approx(s2[0], rel=1e-12)
    assert 4.0 / x ** 2 * s1[0].real == pytest.approx(mie_efficiencies(x, m)[0], rel=1e-12)


def test_oracle_dda_sphere_mueller_matches_mie():
    """16^3 sphere, m = 1.33+0.1i, x = 1: S11 within 2 % of Mie over 0..180 deg
    and the polarisation ratios S12/S11, S33/S11, S34/S11 within 0.01 (so the
    amplitude-matrix basis, sign and phase conventions are those of the exact
    sphere)."""
    n, m, x = 16, 1.33 + 0.1j, 1.0
    prob = targets.make_problem(n, m=m, x=x)
    gp = O.GreenParams(n, n, n, ak=tuple(prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    k = prob.incid[0].k
    aks, em1, em2 = targets.scattering_planes(k, prob.incid[0].e, 10.0, (0.0, 90.0))
    f = []
    for r in range(2):
        b = O.gather_compact(prob.rhs(r), op.occ, prob.nat)
        adia = O.gather_compact(prob.adia(r), op.occ, prob.nat)
        aoff = np.zeros_like(adia)
        res = O.solve_qmrccg(lambda v: op.apply_compact(v, adia, aoff), b, np.zeros_like(b), 1000, 1e-7)
        sc = O.scat(res.x, op.occ, prob.nx, prob.ny, 0, k, aks, (1, 1, 1), em1, em2, 1.0, 0.5, prob.incid[r].e,
                    prob.x0)
        f.append((sc["f1"], sc["f2"]))
    S = O.amplitude_matrix(k, prob.incid[0].e, prob.incid[1].e, em2, f[0][0], f[0][1], f[1][0], f[1][1])
    M = O.mueller_from_amplitude(S)
    theta = np.deg2rad(np.tile(np.arange(0.0, 180.5, 10.0), 2))
    s1, s2 = mie_amplitudes(x, m, theta)
    s11 = 0.5 * (np.abs(s1) ** 2 + np.abs(s2) ** 2)
    s12 = 0.5 * (np.abs(s2) ** 2 - np.abs(s1) ** 2)
    s33 = (s2 * np.conj(s1)).real
    s34 = (s2 * np.conj(s1)).imag
    assert np.max(np.abs(M[:, 0, 0] / s11 - 1.0)) < 0.02
    assert np.max(np.abs(M[:, 0, 1] / M[:, 0, 0] - s12 / s11)) < 0.01
    assert np.max(np.abs(M[:, 2, 2] / M[:, 0, 0] - s33 / s11)) < 0.01
    assert np.max(np.abs(M[:, 2, 3] / M[:, 0, 0] - s34 / s11)) < 0.01
