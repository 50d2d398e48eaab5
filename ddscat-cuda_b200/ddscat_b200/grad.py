"""Gradients of extinction and far-field intensities with respect to the
per-dipole permittivity (thin optional layer over ddscat_b200_adjoint_f32).

The DDA matrix A(eps) = diag(CXADIA(eps)) - G is complex symmetric, so the
derivative of any holomorphic functional F = s^T P of the polarisation P =
A^-1 E costs one adjoint solve A lam = s and a per-site product:
dF/deps_j = -sum_c lam_c(j) dCXADIA_c(j)/deps_j P_c(j).  With the lattice
dispersion relation polarisability (Draine & Goodman 1993)
    1/alpha = (4 pi / 3)(eps + 2)/(eps - 1) + (b1 + eps b2 + eps b3 S)(kd)^2 - (2/3) i (kd)^3
the site derivative is d(1/alpha)/deps = -4 pi/(eps - 1)^2 + (b2 + b3 S)(kd)^2.

* Cext = 4 pi k Im(E^H P)/E02 -> F = conj(E)^T P;
  dCext/dRe eps = 4 pi k Im(g)/E02, dCext/dIm eps = 4 pi k Re(g)/E02.
* A scattering amplitude f_m(n) = |k|^3/sqrt(E02) sum_j e_m . P_j exp(-i k_s . r_j)
  (the normalisation of ddscat_cuda_scat_f32) -> F = w^T P; the intensity
  I = |f_1|^2 + |f_2|^2 has dI = 2 Re(conj(f_1) df_1 + conj(f_2) df_2).

Gradients are returned as (dRe, dIm) pairs per occupied site (compact order);
CextFunction exposes the same through torch.autograd with PyTorch's complex
convention (grad = dL/dRe eps + i dL/dIm eps).
"""
from __future__ import annotations

import math

import numpy as np

from .targets import B1, B2, B3


def ldr_inv_alpha(eps, kd, khat, e):
    """1/alpha_LDR (lattice units) for permittivity eps (array)."""
    eps = np.asarray(eps, dtype=np.complex128)
    S = float(np.sum((np.asarray(khat) * np.real(np.asarray(e))) ** 2))
    return (4.0 * math.pi / 3.0) * (eps + 2.0) / (eps - 1.0) + (B1 + eps * B2 + eps * B3 * S) * kd ** 2 \
        - (2.0 / 3.0) * 1j * kd ** 3


def ldr_dinv_alpha(eps, kd, khat, e):
    """d(1/alpha_LDR)/d eps."""
    eps = np.asarray(eps, dtype=np.complex128)
    S = float(np.sum((np.asarray(khat) * np.real(np.asarray(e))) ** 2))
    return -4.0 * math.pi / (eps - 1.0) ** 2 + (B2 + B3 * S) * kd ** 2


def _full(prob, site_vals, fill):
    """3*NAT vector with site_vals (NAT0, compact order) on occupied sites."""
    v = np.full(prob.nat, fill, dtype=np.complex128)
    v[prob.occ] = site_vals
    return np.tile(v, 3)


def site_inputs(prob, r, eps):
    """(b, CXADIA, dCXADIA/deps) full vectors of RHS r for per-site permittivity eps (NAT0)."""
    inc = prob.incid[r]
    khat = inc.k / np.linalg.norm(inc.k)
    kd = float(np.linalg.norm(inc.k))
    ia = ldr_inv_alpha(eps, kd, khat, inc.e)
    dia = ldr_dinv_alpha(eps, kd, khat, inc.e)
    return prob.rhs(r), _full(prob, ia, ia[0]), _full(prob, dia, 0.0)


def farfield_weights(prob, r, aks, ems, e02=1.0):
    """Full 3*NAT vectors w with f = w^T P for each (scattering wave vector, basis vector)."""
    kk = float(np.linalg.norm(prob.incid[r].k))
    term = kk ** 3 / math.sqrt(e02)
    pos = prob.positions()
    out = []
    for ks, em in zip(aks, ems):
        ph = np.exp(-1j * (pos @ np.asarray(ks, dtype=np.float64))) * (prob.iocc != 0)
        out.append(np.concatenate([term * float(em[c]) * ph for c in range(3)]))
    return out


def _solve(dda, b, adia, tol, maxit):
    x = np.zeros((b.shape[0], b.shape[1]), dtype=np.complex64)
    out = dda.solve_batch("qmrccg", b.astype(np.complex64), x, adia.astype(np.complex64), maxit=maxit, tol=tol,
                          replace=True, symmetric=True)
    return x, out


def cext_and_grad(dda, prob, r, eps, tol=1e-5, maxit=2000, e02=1.0):
    """Cext of RHS r for per-site permittivity eps (NAT0 complex) and its
    gradient (dRe, dIm) per occupied site, FP32 forward and adjoint solves."""
    b, adia, dadia = site_inputs(prob, r, eps)
    x, _ = _solve(dda, b[None, :], adia[None, :], tol, maxit)
    kk = float(np.linalg.norm(prob.incid[r].k))
    cext = 4.0 * math.pi * kk * np.vdot(b.astype(np.complex128), x[0].astype(np.complex128)).imag / e02
    g, _, _, _ = dda.adjoint(x, np.conj(b)[None, :], adia[None, :], dadia[None, :], maxit=maxit, tol=tol)
    gs = g[0][prob.occ].astype(np.complex128)
    fac = 4.0 * math.pi * kk / e02
    return cext, fac * gs.imag, fac * gs.real


def intensity_and_grad(dda, prob, r, eps, aks, em1, em2, tol=1e-5, maxit=2000, e02=1.0):
    """I(n) = |f_1|^2 + |f_2|^2 at each scattering wave vector of aks and its
    gradient (dRe, dIm) per occupied site: arrays (ndir,), (ndir, NAT0), (ndir, NAT0)."""
    b, adia, dadia = site_inputs(prob, r, eps)
    x, _ = _solve(dda, b[None, :], adia[None, :], tol, maxit)
    nd = len(aks)
    w = farfield_weights(prob, r, list(aks) + list(aks), list(em1) + list(em2), e02)
    W = np.stack(w)
    f = W @ x[0].astype(np.complex128)  # f_1 for every direction, then f_2
    R = 2 * nd
    g, _, _, _ = dda.adjoint(np.repeat(x, R, axis=0), W, np.repeat(adia[None, :], R, axis=0),
                             np.repeat(dadia[None, :], R, axis=0), maxit=maxit, tol=tol)
    gs = g[:, prob.occ].astype(np.complex128)
    inten = np.abs(f[:nd]) ** 2 + np.abs(f[nd:]) ** 2
    h = np.conj(f[:nd])[:, None] * gs[:nd] + np.conj(f[nd:])[:, None] * gs[nd:]
    return inten, 2.0 * h.real, -2.0 * h.imag


def cext_function():
    """torch.autograd.Function computing Cext(eps) of one RHS; eps is a
    complex128 tensor of per-site permittivities (NAT0, compact order)."""
    import torch

    class CextFunction(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eps, dda, prob, r):
            e = eps.detach().cpu().numpy()
            cext, gre, gim = cext_and_grad(dda, prob, r, e)
            ctx.save_for_backward(torch.from_numpy(gre + 1j * gim))
            return torch.tensor(cext, dtype=torch.float64)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None, None, None

    return CextFunction
