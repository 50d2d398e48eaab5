"""Polarisability prescriptions of the synthetic inputs (CPU): LATTDR (Draine &
Goodman 1993), GKDLDR (Gutkowicz-Krusin & Draine 2004) and FLTRCD (filtered
coupled dipoles), restated in ddscat_b200.targets from the published formulas.
DDSCAT's own ALPHADIAG is not part of the reference, so these are checked
against the formulas' defining properties and the physics of a lossless
sphere."""
import math

import numpy as np
import pytest

from ddscat_b200 import targets
from oracle import ddscat_oracle as O


def _dirs():
    rng = np.random.default_rng(11)
    k = rng.normal(size=3)
    k /= np.linalg.norm(k)
    e = np.cross(k, rng.normal(size=3))
    return k, e / np.linalg.norm(e)


def test_lattdr_matches_ldr_alpha():
    khat, e = _dirs()
    for m in (1.33 + 0.05j, 1.6 + 0.02j, 2.5 + 1.0j):
        ia = targets.inv_alpha_eps(m * m, 0.4, khat, e, "LATTDR")
        assert np.allclose(ia, 1.0 / targets.ldr_alpha(m, 0.4, khat, e), rtol=1e-13)


def test_gkdldr_is_ldr_with_per_component_shape_factor():
    """Component j of GKDLDR is the LDR formula with S replaced by a_j^2: it
    depends on the propagation direction, not on the polarisation."""
    khat, e = _dirs()
    m, kd = 1.5 + 0.01j, 0.3
    eps = m * m
    ia = targets.inv_alpha_eps(eps, kd, khat, e, "GKDLDR")
    base = (4 * math.pi / 3) * (eps + 2) / (eps - 1) - (2 / 3) * 1j * kd ** 3
    for j in range(3):
        want = base + (targets.B1 + eps * targets.B2 + eps * targets.B3 * khat[j] ** 2) * kd ** 2
        assert ia[j] == pytest.approx(want, rel=1e-13)
    e2 = np.cross(khat, e)
    assert np.allclose(ia, targets.inv_alpha_eps(eps, kd, khat, e2, "GKDLDR"), rtol=1e-14)
    # k along x, e along y: LATTDR's S = 0 equals GKDLDR's transverse components
    ix = targets.inv_alpha_eps(eps, kd, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), "GKDLDR")
    il = targets.inv_alpha_eps(eps, kd, (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), "LATTDR")
    assert ix[1] == pytest.approx(il[1], rel=1e-14) and ix[2] == pytest.approx(il[2], rel=1e-14)
    assert abs(ix[0] - il[0]) > 1e-3 * abs(il[0])


@pytest.mark.parametrize("cmdpol", targets.PRESCRIPTIONS)
def test_clausius_mossotti_limit_and_radiative_reaction(cmdpol):
    """alpha -> alpha_CM as kd -> 0 with an O((kd)^2) correction, and for real m
    Im(1/alpha) = -(2/3)(kd)^3 exactly (the radiative-reaction term that makes a
    lossless dipole lattice conserve energy)."""
    khat, e = _dirs()
    m = 1.7
    eps = m * m
    inv_cm = (4 * math.pi / 3) * (eps + 2) / (eps - 1)
    for kd in (1e-2, 1e-3):
        ia = targets.inv_alpha_eps(eps, kd, khat, e, cmdpol)
        assert np.all(np.abs(ia - inv_cm) <= 5 * kd ** 2 * abs(eps))
    for kd in (0.2, 0.7):
        ia = targets.inv_alpha_eps(eps, kd, khat, e, cmdpol)
        assert np.allclose(ia.imag, -(2 / 3) * kd ** 3, rtol=1e-12, atol=0)


def test_fltrcd_formula():
    khat, e = _dirs()
    eps, kd = (1.33 + 0.01j) ** 2, 0.5
    ia = targets.inv_alpha_eps(eps, kd, khat, e, "FLTRCD")
    want = ((4 * math.pi / 3) * (eps + 2) / (eps - 1) - (4 / 3) * kd ** 2
            - (2 / (3 * math.pi)) * math.log((math.pi - kd) / (math.pi + kd)) * kd ** 3 - (2 / 3) * 1j * kd ** 3)
    assert np.allclose(ia, want, rtol=1e-14)
    with pytest.raises(ValueError):
        targets.inv_alpha_eps(eps, 3.2, khat, e, "FLTRCD")
    with pytest.raises(ValueError):
        targets.make_problem(4, cmdpol="NOSUCH")


@pytest.mark.parametrize("cmdpol", targets.PRESCRIPTIONS)
def test_lossless_sphere_absorbs_nothing(cmdpol):
    """Real refractive index: with Im(1/alpha) = -(2/3)(kd)^3 the DDA's
    absorption cross section (EVALQ's Cabs) vanishes and Cext = Csca
    (optical theorem), whatever the prescription's real part."""
    n = 8
    prob = targets.make_problem(n, m=1.4 + 0.0j, x=1.5, cmdpol=cmdpol)
    k = prob.incid[0].k
    op = O.Operator.from_params(O.GreenParams(n, n, n, ak=tuple(k)), prob.iocc)
    occ = op.occ
    b = O.gather_compact(prob.rhs(0), occ, prob.nat).astype(np.complex128)
    adia = prob.adia(0)
    assert not np.allclose(adia[:prob.nat], adia[prob.nat:2 * prob.nat]) or cmdpol != "GKDLDR"
    ac = O.gather_compact(adia, occ, prob.nat).astype(np.complex128)
    zero = np.zeros_like(ac)
    res = O.solve_qmrccg(lambda v: op.apply_compact(v, ac, zero), b, np.zeros_like(b), 500, 1e-12)
    cabs, cext, _ = O.evalq(b, res.x, ac, zero, k, 1.0)
    assert abs(cabs) <= 1e-8 * cext
    sc = O.scat(res.x, occ, n, n, 0, k, np.zeros((0, 3)), (1.0, 1.0, 1.0), None, None, 1.0, 0.5, prob.incid[0].e,
                prob.x0)
    assert sc["csca"] == pytest.approx(cext, rel=2e-2)  # quadrature error of SCAT's angular integration
