"""Gradients of extinction and far-field intensities with respect to the
per-dipole permittivity (thin optional layer over ddscat_b200_adjoint_f32).

The DDA matrix A(eps) = diag(CXADIA(eps)) - G is complex symmetric, so the
derivative of any holomorphic functional F = s^T P of the polarisation P =
A^-1 E costs one adjoint solve A lam = s and a per-site product:
dF/deps_j = -sum_c lam_c(j) dCXADIA_c(j)/deps_j P_c(j).  With the lattice
dispersion relation polarisabilities (Draine & Goodman 1993; the per-component
form of Gutkowicz-Krusin & Draine 2004)
    1/alpha_c = (4 pi / 3)(eps + 2)/(eps - 1) + (b1 + eps b2 + eps b3 S_c)(kd)^2 - (2/3) i (kd)^3
the site derivative is d(1/alpha_c)/deps = -4 pi/(eps - 1)^2 + (b2 + b3 S_c)(kd)^2
(S_c = sum_j (a_j e_j)^2 for LATTDR, a_c^2 for GKDLDR); the filtered coupled
dipole form (FLTRCD) has only the first term.  The problem's prescription
(Problem.cmdpol) is used.

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

from .targets import B1, B2, B3, dinv_alpha_deps, inv_alpha_eps


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
    """3*NAT vector with site_vals ((3, NAT0): per component, compact order) on
    occupied sites and fill[c] on vacuum sites."""
    v = np.empty((3, prob.nat), dtype=np.complex128)
    for c in range(3):
        v[c] = fill[c]
        v[c, prob.occ] = site_vals[c]
    return v.reshape(-1)


def site_inputs(prob, r, eps):
    """(b, CXADIA, dCXADIA/deps) full vectors of RHS r for per-site permittivity
    eps (NAT0), with the problem's polarisability prescription."""
    inc = prob.incid[r]
    khat = inc.k / np.linalg.norm(inc.k)
    kd = float(np.linalg.norm(inc.k))
    cmdpol = getattr(prob, "cmdpol", "LATTDR")
    ia = inv_alpha_eps(eps, kd, khat, inc.e, cmdpol)
    dia = dinv_alpha_deps(eps, kd, khat, inc.e, cmdpol)
    return prob.rhs(r), _full(prob, ia, ia[:, 0]), _full(prob, dia, np.zeros(3))


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


def _on_gpu(dda):
    """Device tensors for the adjoint inputs when torch has a CUDA device and
    the library object is the real one (it takes device pointers)."""
    if not getattr(dda, "takes_device_pointers", False):
        return None
    try:
        import torch
    except ImportError:
        return None
    return torch if torch.cuda.is_available() else None


def cext_and_grad(dda, prob, r, eps, tol=1e-5, maxit=2000, e02=1.0):
    """Cext of RHS r for per-site permittivity eps (NAT0 complex) and its
    gradient (dRe, dIm) per occupied site: FP32 forward and adjoint solves in
    one call (ddscat_b200_adjoint_fwd_f32, which recomputes the forward field
    instead of taking it from the caller)."""
    b, adia, dadia = site_inputs(prob, r, eps)
    b64, a64, d64 = (v.astype(np.complex64) for v in (b, adia, dadia))
    src = np.conj(b64)[None, :]
    torch = _on_gpu(dda)
    if torch is not None:
        dev = torch.device("cuda", torch.cuda.current_device())
        t = lambda v: torch.from_numpy(np.ascontiguousarray(v)).to(dev)  # noqa: E731
        g, p, _, _ = dda.adjoint_fwd(t(b64), t(src), t(a64), t(d64), maxit=maxit, tol=tol, want_p=True)
        g, p = g.cpu().numpy(), p.cpu().numpy()
    else:
        g, p, _, _ = dda.adjoint_fwd(b64, src, a64, d64, maxit=maxit, tol=tol, want_p=True)
    kk = float(np.linalg.norm(prob.incid[r].k))
    cext = 4.0 * math.pi * kk * np.vdot(b.astype(np.complex128), p.astype(np.complex128)).imag / e02
    gs = g[0][prob.occ].astype(np.complex128)
    fac = 4.0 * math.pi * kk / e02
    return cext, fac * gs.imag, fac * gs.real


def intensity_and_grad(dda, prob, r, eps, aks, em1, em2, tol=1e-5, maxit=2000, e02=1.0):
    """I(n) = |f_1|^2 + |f_2|^2 at each scattering wave vector of aks and its
    gradient (dRe, dIm) per occupied site: arrays (ndir,), (ndir, NAT0), (ndir, NAT0).
    The far-field adjoint sources are built by the library
    (ddscat_b200_ffweights_f32; on the GPU, in device memory when torch has a
    CUDA device) and the forward field is recomputed inside the adjoint call."""
    b, adia, dadia = site_inputs(prob, r, eps)
    b64, a64, d64 = (v.astype(np.complex64) for v in (b, adia, dadia))
    nd = len(aks)
    aks2 = np.concatenate([np.asarray(aks, dtype=np.float64)] * 2)
    ems = np.concatenate([np.asarray(em1, dtype=np.float64), np.asarray(em2, dtype=np.float64)])
    torch = _on_gpu(dda)
    if torch is not None:
        dev = torch.device("cuda", torch.cuda.current_device())
        W = torch.empty((2 * nd, 3 * prob.nat), dtype=torch.complex64, device=dev)
        dda.ffweights(aks2, ems, prob.x0, e02, out=W)
        t = lambda v: torch.from_numpy(np.ascontiguousarray(v)).to(dev)  # noqa: E731
        g, p, _, _ = dda.adjoint_fwd(t(b64), W, t(a64), t(d64), maxit=maxit, tol=tol, want_p=True)
        f = (W.to(torch.complex128) @ p.to(torch.complex128)).cpu().numpy()  # f_1 for every direction, then f_2
        gs = g[:, torch.from_numpy(prob.occ).to(dev)].to(torch.complex128).cpu().numpy()
    else:
        W = dda.ffweights(aks2, ems, prob.x0, e02)
        g, p, _, _ = dda.adjoint_fwd(b64, W, a64, d64, maxit=maxit, tol=tol, want_p=True)
        f = W.astype(np.complex128) @ p.astype(np.complex128)
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
