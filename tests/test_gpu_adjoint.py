"""Adjoint gradients (ddscat_b200_adjoint_f32 and ddscat_b200.grad) on the C5a
configuration: a 48^3 two-material voxel target (occupancy 0.6 from a seed;
material 1 m = 1.5+0.01i, material 2 m = 1.2), x = 8.

* dCext/deps from FP32 forward + adjoint solves against the FP64 reference
  gradient (FP64 forward and adjoint solves, complex-double inputs): <= 1e-3
  of the largest site derivative;
* the FP64 gradient against central finite differences (step 1e-3 in Re eps
  and Im eps, FP64 solves, Cext evaluated in FP64) on 50 random dipoles: <=
  1e-3 relative, and the FP32 gradient against the same differences;
* the intensity |f_1|^2 + |f_2|^2 at 10 fixed scattering angles: FP32 adjoint
  gradient against finite differences on 5 dipoles;
* torch.autograd through CextFunction returns dCext/dRe eps + i dCext/dIm eps."""
import math

import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import grad as G
from ddscat_b200 import targets

H = 1e-3


def _setup():
    prob, mat = targets.voxel_problem(48, p_occ=0.6, m1=1.5 + 0.01j, m2=1.2 + 0.0j, x=8.0, seed=0)
    eps = np.where(mat[prob.occ] == 1, (1.5 + 0.01j) ** 2, (1.2 + 0.0j) ** 2).astype(np.complex128)
    dda = D.DDA()
    dda.prepare_green(48, 48, 48, prob.iocc, prob.incid[0].k)
    return prob, eps, dda


def _fd_batch(prob, eps, sites, r=0):
    """Full adia vectors for eps perturbed by +-H and +-iH at each site."""
    rows = []
    for s in sites:
        for d in (H, -H, 1j * H, -1j * H):
            e2 = eps.copy()
            e2[s] += d
            rows.append(G.site_inputs(prob, r, e2)[1])
    return np.stack(rows)


def _solve64(dda, b, adia, tol=1e-12):
    x = np.zeros(b.shape, dtype=np.complex128)
    out = dda.solve_batch_f64("qmrccg", b, x, adia, maxit=4000, tol=tol, replace=True, symmetric=True)
    assert np.all(out.status == 0)
    return x


@pytest.mark.gpu
def test_c5a_cext_gradient():
    prob, eps, dda = _setup()
    kk = float(np.linalg.norm(prob.incid[0].k))
    fac = 4.0 * math.pi * kk
    cext, gre, gim = G.cext_and_grad(dda, prob, 0, eps)
    b, adia, dadia = G.site_inputs(prob, 0, eps)
    b64 = b.astype(np.complex128)[None, :]
    x64 = _solve64(dda, b64, adia[None, :])
    lam = _solve64(dda, np.conj(b64), adia[None, :])
    occ3 = np.concatenate([prob.occ + c * prob.nat for c in range(3)])
    g64 = -np.sum((lam[0][occ3] * dadia[occ3] * x64[0][occ3]).reshape(3, -1), axis=0)
    gre64, gim64 = fac * g64.imag, fac * g64.real
    c64 = fac * np.vdot(b64[0], x64[0]).imag
    assert abs(cext - c64) <= 1e-4 * abs(c64)
    scale = max(np.abs(gre64).max(), np.abs(gim64).max())
    assert np.abs(gre - gre64).max() <= 1e-3 * scale and np.abs(gim - gim64).max() <= 1e-3 * scale
    # central differences on 50 random dipoles (200 FP64 solves in one batch)
    rng = np.random.default_rng(1)
    sites = rng.choice(prob.nat0, size=50, replace=False)
    A = _fd_batch(prob, eps, sites)
    X = _solve64(dda, np.repeat(b64, A.shape[0], axis=0), A)
    C = fac * np.einsum("j,rj->r", np.conj(b64[0]), X).imag
    C = C.reshape(len(sites), 4)
    fd_re = (C[:, 0] - C[:, 1]) / (2 * H)
    fd_im = (C[:, 2] - C[:, 3]) / (2 * H)
    sc = max(np.abs(fd_re).max(), np.abs(fd_im).max())
    assert np.abs(gre64[sites] - fd_re).max() <= 1e-3 * sc
    assert np.abs(gim64[sites] - fd_im).max() <= 1e-3 * sc
    assert np.abs(gre[sites] - fd_re).max() <= 1e-3 * sc
    assert np.abs(gim[sites] - fd_im).max() <= 1e-3 * sc
    dda.release()


@pytest.mark.gpu
def test_c5a_intensity_gradient():
    prob, eps, dda = _setup()
    k = prob.incid[0].k
    kk = float(np.linalg.norm(k))
    aks, em1, em2 = [], [], []
    for t in np.deg2rad(np.linspace(10.0, 170.0, 10)):  # 10 fixed angles in the x-y plane
        n = np.array([math.cos(t), math.sin(t), 0.0])
        e1 = np.array([-math.sin(t), math.cos(t), 0.0])
        aks.append(kk * n)
        em1.append(e1)
        em2.append(np.cross(n, e1))
    inten, gre, gim = G.intensity_and_grad(dda, prob, 0, eps, aks, em1, em2)
    rng = np.random.default_rng(2)
    sites = rng.choice(prob.nat0, size=5, replace=False)
    A = _fd_batch(prob, eps, sites)
    b64 = prob.rhs(0).astype(np.complex128)[None, :]
    X = _solve64(dda, np.repeat(b64, A.shape[0], axis=0), A)
    W = np.stack(G.farfield_weights(prob, 0, aks + aks, em1 + em2))
    F = X @ W.T  # (4*5, 20)
    I = np.abs(F[:, :10]) ** 2 + np.abs(F[:, 10:]) ** 2
    I = I.reshape(len(sites), 4, 10)
    fd_re = (I[:, 0] - I[:, 1]) / (2 * H)
    fd_im = (I[:, 2] - I[:, 3]) / (2 * H)
    for d in range(10):
        sc = max(np.abs(fd_re[:, d]).max(), np.abs(fd_im[:, d]).max())
        assert np.abs(gre[d, sites] - fd_re[:, d]).max() <= 1e-3 * sc, d
        assert np.abs(gim[d, sites] - fd_im[:, d]).max() <= 1e-3 * sc, d
    dda.release()


@pytest.mark.gpu
def test_cext_autograd():
    torch = pytest.importorskip("torch")
    n = 10
    prob, mat = targets.voxel_problem(n, x=2.0, seed=3)
    eps0 = np.where(mat[prob.occ] == 1, (1.5 + 0.01j) ** 2, 1.44 + 0j).astype(np.complex128)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    eps = torch.tensor(eps0, requires_grad=True)
    Cext = G.cext_function()
    c = Cext.apply(eps, dda, prob, 0)
    (g,) = torch.autograd.grad(c, eps)
    _, gre, gim = G.cext_and_grad(dda, prob, 0, eps0)
    assert np.allclose(g.numpy().real, gre) and np.allclose(g.numpy().imag, gim)
    dda.release()


@pytest.mark.gpu
def test_ffweights_and_recomputed_forward_adjoint():
    """ddscat_b200_ffweights_f32 equals the host restatement of the far-field
    weights (1e-6 of max |w|, host and device outputs), and the adjoint with
    the forward field recomputed inside the call (ddscat_b200_adjoint_fwd_f32)
    gives the gradient of the adjoint with a caller-held forward solution
    (ddscat_b200_adjoint_f32) to 1e-4 of its largest entry."""
    torch = pytest.importorskip("torch")
    n = 12
    prob, mat = targets.voxel_problem(n, x=2.0, seed=5)
    eps = np.where(mat[prob.occ] == 1, (1.5 + 0.01j) ** 2, (1.2 + 0.0j) ** 2).astype(np.complex128)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    k = prob.incid[0].k
    aks, em1, em2 = targets.scattering_planes(k, prob.incid[0].e, 45.0, (0.0,))
    aks2, ems = np.concatenate([aks, aks]), np.concatenate([em1, em2])
    W = dda.ffweights(aks2, ems, prob.x0)
    Wh = np.stack(G.farfield_weights(prob, 0, list(aks2), list(ems)))
    assert np.abs(W - Wh).max() <= 1e-6 * np.abs(Wh).max()
    Wd = torch.empty(W.shape, dtype=torch.complex64, device="cuda")
    dda.ffweights(aks2, ems, prob.x0, out=Wd)
    assert np.abs(Wd.cpu().numpy() - Wh).max() <= 1e-6 * np.abs(Wh).max()
    b, adia, dadia = (v.astype(np.complex64) for v in G.site_inputs(prob, 0, eps))
    g2, p, it, tole = dda.adjoint_fwd(b, W, adia, dadia, maxit=2000, tol=1e-6, want_p=True)
    assert it.shape == (W.shape[0] + 1,) and np.all(tole <= 1e-6)
    R = W.shape[0]
    g1, _, _, _ = dda.adjoint(np.repeat(p[None, :], R, axis=0), W, np.repeat(adia[None, :], R, axis=0),
                              np.repeat(dadia[None, :], R, axis=0), maxit=2000, tol=1e-6)
    assert np.abs(g2 - g1).max() <= 1e-4 * np.abs(g1).max()
    assert np.all(g2[:, prob.iocc == 0] == 0)
    dda.release()
