"""CPU checks of the oracle's radiative-torque restatement (DDSCAT's DOTORQ).

1. The scattered angular-momentum flux, integrated over the far field, equals
   minus the torque that the dipoles' own fields (the fields of the other
   dipoles plus each dipole's radiation reaction) exert on them -- angular
   momentum conservation for an arbitrary set of oscillating dipoles, checked
   with analytic dipole fields and central-difference field gradients.
2. Solved DDA spheres: in circularly polarised light the net torque along k is
   C_abs (one hbar per absorbed photon), zero for a lossless sphere, and zero in
   linearly polarised light (mirror symmetry); the tolerances are the
   quadrature error of SCAT's ETASCA = 0.5 direction set."""
import math

import numpy as np
import pytest
import scipy.sparse.linalg as sla

from ddscat_b200 import targets
from oracle import ddscat_oracle as O


def _dipole_field(rr, rl, p, k):
    R = rr - rl
    d = np.linalg.norm(R)
    n = R / d
    return np.exp(1j * k * d) * (k * k * (p - n * (n @ p)) / d + (3 * n * (n @ p) - p) * (1 / d ** 3 - 1j * k / d ** 2))


def test_flux_equals_near_field_torque():
    rng = np.random.default_rng(3)
    k, nd = 1.3, 12
    r = rng.normal(size=(nd, 3)) * 1.2
    P = rng.normal(size=(nd, 3)) + 1j * rng.normal(size=(nd, 3))

    def others(j, rr):
        return sum(_dipole_field(rr, r[l], P[l], k) for l in range(nd) if l != j)

    near = np.zeros(3)
    h = 1e-5
    for j in range(nd):
        e = others(j, r[j]) + (2.0 / 3.0) * 1j * k ** 3 * P[j]  # radiation reaction of j itself
        grad = np.zeros((3, 3), dtype=complex)
        for i in range(3):
            dr = np.zeros(3)
            dr[i] = h
            grad[i] = (others(j, r[j] + dr) - others(j, r[j] - dr)) / (2 * h)
        force = 0.5 * np.real(grad @ np.conj(P[j]))
        near -= 0.5 * np.real(np.cross(P[j], np.conj(e))) + np.cross(r[j], force)
    x, wx = np.polynomial.legendre.leggauss(100)
    nph = 200
    phi = (np.arange(nph) + 0.5) * 2 * np.pi / nph
    ct = np.repeat(x, nph)
    st = np.sqrt(1 - ct ** 2)
    ph = np.tile(phi, 100)
    n = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=1)
    w = np.repeat(wx, nph) * (2 * np.pi / nph)
    S, U = O.torque_flux_sums(P.T.reshape(-1), r, n * k)
    far = k ** 3 / (8 * np.pi) * (w @ O.torque_flux_integrand(n, S, U, k))
    assert np.linalg.norm(far - near) <= 1e-8 * np.linalg.norm(near)


def _sphere_torque(m, e01, n=10, x=1.5):
    prob = targets.make_problem(n, m=m, x=x)
    k = prob.incid[0].k
    e01 = np.asarray(e01, dtype=np.complex128)
    prob.incid = [targets.Incidence(k=k, e=e01)]
    occ = prob.occ
    b = O.gather_compact(prob.rhs(0).astype(np.complex128), occ, prob.nat)
    a = O.gather_compact(prob.adia(0).astype(np.complex128), occ, prob.nat)
    op = O.Operator.from_params(O.GreenParams(n, n, n, ak=tuple(k)), prob.iocc)
    z = np.zeros_like(a)
    L = sla.LinearOperator((b.size, b.size), matvec=lambda v: op.apply_compact(v, a, z), dtype=np.complex128)
    p, info = sla.gmres(L, b, rtol=1e-11, restart=200, maxiter=2000)
    assert info == 0
    e02 = float(np.real(np.vdot(e01, e01)))
    cabs, cext, _ = O.evalq(b, p, a, z, k, e02)
    out = O.scat_torque(p, b, occ, n, n, k, (1, 1, 1), e02, 0.5, e01, prob.x0)
    return out, cabs, cext, k / np.linalg.norm(k)


@pytest.mark.parametrize("m", [1.5 + 0.1j, 1.5 + 0.0j])
def test_sphere_circular_torque_is_absorbed_spin(m):
    s = 1 / math.sqrt(2)
    out, cabs, cext, khat = _sphere_torque(m, [0, s, 1j * s])
    net = out["ctrq"]
    assert abs(net @ khat - cabs) <= 3e-3 * cext
    assert np.linalg.norm(net - (net @ khat) * khat) <= 1e-6 * cext


def test_sphere_linear_torque_vanishes():
    out, cabs, cext, khat = _sphere_torque(1.5 + 0.1j, [0, 1, 0])
    assert np.abs(out["ctrq"]).max() <= 1e-6 * cext
