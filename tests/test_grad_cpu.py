"""CPU check of the gradient layer (ddscat_b200/grad.py): the LDR derivative,
the site inputs, the far-field weights and the chain rules of cext_and_grad
and intensity_and_grad, run against an FP64 oracle stand-in for the library
(solve_batch and the adjoint entry point restated from their C-ABI contract,
include/ddscat_b200.h) and compared with central finite differences of the
oracle's EVALQ and SCAT."""
import math

import numpy as np
import pytest

from ddscat_b200 import grad as G
from ddscat_b200 import targets
from oracle import ddscat_oracle as O


class OracleDDA:
    """FP64 stand-ins for DDA.solve_batch and DDA.adjoint of one prepared target."""

    def __init__(self, prob):
        self.prob = prob
        gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(prob.incid[0].k))
        self.op = O.Operator.from_params(gp, prob.iocc)

    def _solve(self, b, adia):
        occ, nat = self.op.occ, self.prob.nat
        bc = O.gather_compact(b.astype(np.complex128), occ, nat)
        ac = O.gather_compact(adia.astype(np.complex128), occ, nat)
        zero = np.zeros_like(ac)
        res = O.solve_qmrccg(lambda v: self.op.apply_compact(v, ac, zero), bc, np.zeros_like(bc), 2000, 1e-12)
        assert res.status == 0
        return O.scatter_full(res.x, occ, nat)

    def solve_batch(self, name, b, x, adia, maxit=300, tol=1e-5, replace=False, symmetric=False):
        for r in range(b.shape[0]):
            x[r] = self._solve(b[r], adia[r])
        return None

    def adjoint_fwd(self, e, src, adia, dadia, maxit=1000, tol=1e-5, want_p=False):
        """ddscat_b200_adjoint_fwd_f32: the forward solution of A P = e is
        recomputed inside; grad[k][j] = -sum_c lam_k[c][j] dadia[c][j] P[c][j]."""
        p = self._solve(e, adia)
        nat = self.prob.nat
        out = np.zeros((src.shape[0], nat), dtype=np.complex128)
        for k in range(src.shape[0]):
            lam = self._solve(src[k], adia)
            t = -(lam * dadia.astype(np.complex128) * p).reshape(3, nat)
            out[k] = t.sum(axis=0)
        return out, (p if want_p else None), None, None

    def ffweights(self, aks, ems, x0, e02=1.0, out=None):
        """ddscat_b200_ffweights_f32: w_k = |aks_k|^3/sqrt(E02) em_k exp(-i aks_k . r_j)."""
        return np.stack(G.farfield_weights(self.prob, 0, list(aks), list(ems), e02))

    def adjoint(self, p, src, adia, dadia, maxit=1000, tol=1e-5):
        """grad[r][j] = -sum_c lam[c][j] dadia[c][j] p[c][j], A lam = src (A^T = A)."""
        nat = self.prob.nat
        out = np.zeros((p.shape[0], nat), dtype=np.complex128)
        for r in range(p.shape[0]):
            lam = self._solve(src[r], adia[r])
            t = -(lam * dadia[r].astype(np.complex128) * p[r].astype(np.complex128)).reshape(3, nat)
            out[r] = t.sum(axis=0)
        return out, None, None, None


def _problem():
    prob = targets.make_problem(8, m=1.5 + 0.02j, x=1.2)
    rng = np.random.default_rng(4)
    eps0 = (1.5 + 0.02j) ** 2 + 0.05 * (rng.normal(size=prob.nat0) + 1j * rng.normal(size=prob.nat0))
    return prob, eps0


def test_ldr_derivative_matches_finite_difference():
    prob, eps0 = _problem()
    inc = prob.incid[0]
    khat = inc.k / np.linalg.norm(inc.k)
    kd = float(np.linalg.norm(inc.k))
    h = 1e-6
    fd = (G.ldr_inv_alpha(eps0 + h, kd, khat, inc.e) - G.ldr_inv_alpha(eps0 - h, kd, khat, inc.e)) / (2 * h)
    fdi = (G.ldr_inv_alpha(eps0 + 1j * h, kd, khat, inc.e) - G.ldr_inv_alpha(eps0 - 1j * h, kd, khat, inc.e)) / (2j * h)
    an = G.ldr_dinv_alpha(eps0, kd, khat, inc.e)
    assert np.allclose(fd, an, rtol=1e-7) and np.allclose(fdi, an, rtol=1e-7)  # holomorphic in eps


@pytest.mark.parametrize("cmdpol", targets.PRESCRIPTIONS)
def test_prescription_derivative_matches_finite_difference(cmdpol):
    prob, eps0 = _problem()
    inc = prob.incid[0]
    khat = inc.k / np.linalg.norm(inc.k)
    kd = float(np.linalg.norm(inc.k))
    f = lambda e: targets.inv_alpha_eps(e, kd, khat, inc.e, cmdpol)  # noqa: E731
    h = 1e-6
    fd = (f(eps0 + h) - f(eps0 - h)) / (2 * h)
    fdi = (f(eps0 + 1j * h) - f(eps0 - 1j * h)) / (2j * h)
    an = targets.dinv_alpha_deps(eps0, kd, khat, inc.e, cmdpol)
    assert an.shape == (3, eps0.size)
    assert np.allclose(fd, an, rtol=1e-7) and np.allclose(fdi, an, rtol=1e-7)


def _cext(dda, prob, eps):
    b, adia, _ = G.site_inputs(prob, 0, eps)
    x = dda._solve(b, adia)
    kk = float(np.linalg.norm(prob.incid[0].k))
    occ, nat = dda.op.occ, prob.nat
    ac = O.gather_compact(adia, occ, nat)
    cabs, cext, _ = O.evalq(O.gather_compact(b, occ, nat), O.gather_compact(x, occ, nat), ac, np.zeros_like(ac),
                            prob.incid[0].k, 1.0)
    assert cext == pytest.approx(4 * math.pi * kk * np.vdot(b, x).imag, rel=1e-9)
    return cext


@pytest.mark.parametrize("site", [0, 57, 131])
def test_cext_gradient_matches_finite_difference(site):
    prob, eps0 = _problem()
    dda = OracleDDA(prob)
    c0, gre, gim = G.cext_and_grad(dda, prob, 0, eps0)
    assert c0 == pytest.approx(_cext(dda, prob, eps0), rel=1e-5)
    h = 1e-4
    for d, g in ((h, gre[site]), (1j * h, gim[site])):
        ep, em = eps0.copy(), eps0.copy()
        ep[site] += d
        em[site] -= d
        fd = (_cext(dda, prob, ep) - _cext(dda, prob, em)) / (2 * h)
        assert g == pytest.approx(fd, rel=2e-3, abs=1e-6 * abs(c0))


def test_intensity_gradient_matches_finite_difference():
    prob, eps0 = _problem()
    dda = OracleDDA(prob)
    k = prob.incid[0].k
    aks, em1, em2 = targets.scattering_planes(k, prob.incid[0].e, 60.0, (0.0,))
    inten, gre, gim = G.intensity_and_grad(dda, prob, 0, eps0, aks, em1, em2)

    def scat_intensity(eps):
        b, adia, _ = G.site_inputs(prob, 0, eps)
        x = O.gather_compact(dda._solve(b, adia), dda.op.occ, prob.nat)
        sc = O.scat(x, dda.op.occ, prob.nx, prob.ny, 0, k, aks, (1, 1, 1), em1, em2, 1.0, 0.5, prob.incid[0].e,
                    prob.x0)
        return np.abs(sc["f1"]) ** 2 + np.abs(sc["f2"]) ** 2

    assert np.allclose(inten, scat_intensity(eps0), rtol=1e-4)
    h = 1e-4
    for site in (3, 101):
        for d, g in ((h, gre[:, site]), (1j * h, gim[:, site])):
            ep, em = eps0.copy(), eps0.copy()
            ep[site] += d
            em[site] -= d
            fd = (scat_intensity(ep) - scat_intensity(em)) / (2 * h)
            assert np.allclose(g, fd, rtol=5e-3, atol=1e-5 * inten.max())
