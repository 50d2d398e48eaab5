"""GPU generation of right-hand sides and CXADIA (ddscat_b200_make_inputs_f32,
ddscat_b200_make_inputs_pol_f32) against the host restatement in
ddscat_b200.targets (incident plane wave e0 exp(i k.r_j) and the LATTDR,
GKDLDR and FLTRCD polarisabilities).
Tolerance: 1e-6 of max |value| (both evaluate the formulas in FP64 and round
to complex64)."""
import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets


def _tol(a, b):
    return np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dims,cmdpol", [((16, 16, 16), "GKDLDR"), ((12, 10, 9), "LATTDR"), ((12, 10, 9), "GKDLDR"),
                                         ((16, 16, 16), "FLTRCD")])
def test_make_inputs_matches_host(dims, cmdpol):
    torch = pytest.importorskip("torch")
    nx, ny, nz = dims
    prob = targets.make_problem(nx, ny, nz, m=1.6 + 0.02j, x=4.0, semi=(nx / 2, 0.8 * ny / 2, 0.6 * nz / 2),
                                orientations=targets.random_orientations(3, seed=4), cmdpol=cmdpol)
    R = len(prob.incid)
    ks = np.array([inc.k for inc in prob.incid])
    es = np.array([inc.e for inc in prob.incid])
    dda = D.DDA()
    dda.prepare_green(nx, ny, nz, prob.iocc, prob.incid[0].k)
    b, a = dda.make_inputs(ks, es, prob.x0, prob.m, cmdpol=cmdpol)
    bref = np.stack([prob.rhs(r) for r in range(R)])
    aref = np.stack([prob.adia(r) for r in range(R)])
    assert _tol(b, bref) and _tol(a, aref)
    bd = torch.zeros((R, 3 * prob.nat), dtype=torch.complex64, device="cuda")
    ad = torch.zeros_like(bd)
    dda.make_inputs(ks, es, prob.x0, prob.m, b=bd, adia=ad, cmdpol=cmdpol)
    assert _tol(bd.cpu().numpy(), bref) and _tol(ad.cpu().numpy(), aref)
    # the generated inputs drive a batched solve directly on the device
    xd = torch.zeros_like(bd)
    out = dda.solve_batch("qmrccg", bd, xd, ad, maxit=500, tol=1e-5)
    assert np.all(out.status == 0) and np.all(out.tole <= 1e-5)
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("cmdpol", ["LATTDR", "GKDLDR"])
def test_make_inputs_two_materials(cmdpol):
    n = 12
    prob, mat = targets.voxel_problem(n, m1=1.5 + 0.01j, m2=1.2 + 0.0j, x=3.0, seed=2, cmdpol=cmdpol)
    inc = prob.incid[0]
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, inc.k)
    ms = [1.5 + 0.01j, 1.2 + 0.0j]
    b, a = dda.make_inputs(inc.k[None, :], inc.e[None, :], prob.x0, ms, icomp=mat, cmdpol=cmdpol)
    khat = inc.k / np.linalg.norm(inc.k)
    ia = [targets.inv_alpha_eps(mm * mm, prob.kd, khat, inc.e, cmdpol) for mm in ms]  # (3,) each
    site = np.stack([np.where(mat == 2, ia[1][c], ia[0][c]) for c in range(3)]).astype(np.complex64).reshape(-1)
    assert _tol(a[0], site) and _tol(b[0], prob.rhs(0))
    bad = mat.copy()
    bad[np.flatnonzero(mat)[0]] = 3
    with pytest.raises(D.DDSCATError) as ei:
        dda.make_inputs(inc.k[None, :], inc.e[None, :], prob.x0, ms, icomp=bad)
    assert ei.value.code == 611
    dda.release()


@pytest.mark.gpu
def test_make_inputs_rejects_bad_prescription():
    n = 8
    prob = targets.make_problem(n, x=1.0)
    inc = prob.incid[0]
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, inc.k)
    fx = lambda pol, k: dda.lib.ddscat_b200_make_inputs_pol_f32(  # noqa: E731
        pol, 1, D._ptr(np.asarray(k, dtype=np.float32)), D._ptr(inc.e.astype(np.complex64)),
        D._ptr(np.asarray(prob.x0, dtype=np.float32)), 1, D._ptr(np.array([1.5 + 0.01j], dtype=np.complex64)), None,
        D._ptr(np.zeros(3 * prob.nat, dtype=np.complex64)), None)
    assert fx(7, inc.k) == 610
    assert fx(2, np.array([3.3, 0.0, 0.0])) == 610  # FLTRCD needs kd < pi
    assert fx(2, inc.k) == 0
    dda.release()
