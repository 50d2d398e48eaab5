"""GPU tests of the batched multi-RHS solve (ddscat_b200_solve_batch_f32) and
the all-FP64 residual check (ddscat_b200_residual_f64).

Each RHS of a batch must behave like the single-RHS entry point of the same
solver: TOLE <= TOL, iteration count within max(1, 10 %) of the single solve
(reductions are grouped differently, so the last bit can differ), solution
within 20*TOL, and an FP64 true residual <= 1.2*TOL."""
import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets
from oracle import ddscat_oracle as O

TOL = 1e-5


def _batch_inputs(prob):
    R = len(prob.incid)
    b = np.stack([prob.rhs(r) for r in range(R)])
    adia = np.stack([prob.adia(r) for r in range(R)])
    return b, adia


@pytest.mark.gpu
@pytest.mark.parametrize("n", [12, 16])
@pytest.mark.parametrize("name", ["qmrccg", "pbcgs2"])
def test_batch_matches_single(name, n):
    orients = targets.random_orientations(3, seed=1)
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=2.0, semi=(n / 2, 0.8 * n / 2, 0.6 * n / 2),
                                orientations=orients)
    R = len(prob.incid)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    x = np.zeros_like(b)
    out = dda.solve_batch(name, b, x, adia, None, maxit=400, tol=TOL)
    assert np.all(out.status == 0)
    assert np.all(out.tole <= TOL)
    res64 = dda.residual_f64(b, x, adia)
    assert np.all(res64 <= 1.2 * TOL), res64
    for r in range(R):
        single = dda.solve(name, b[r], adia[r], prob.aoff(), maxit=400, tol=TOL)
        assert abs(single.itno - out.itno[r]) <= max(1, 0.1 * single.itno), (r, single.itno, out.itno[r])
        assert np.linalg.norm(single.x - x[r]) / np.linalg.norm(single.x) < 20 * TOL
    ms, rhs, calls = dda.last_solve_stats()
    assert rhs == int(out.ncompte.sum()) and calls > 0 and ms > 0
    dda.release()


@pytest.mark.gpu
def test_batch_device_pointers_and_breakdown_mask():
    torch = pytest.importorskip("torch")
    n = 16
    prob = targets.make_problem(n, m=1.5 + 0.01j, x=2.0, orientations=targets.random_orientations(2, seed=3))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    b[1] = 0  # a zero right-hand side is rejected for that RHS only (QMRCCG code 52)
    xh = np.zeros_like(b)
    host = dda.solve_batch("qmrccg", b, xh, adia, maxit=300, tol=TOL)
    assert host.status[1] == 52 and np.all(np.delete(host.status, 1) == 0)
    bd = torch.from_numpy(b).cuda()
    ad = torch.from_numpy(adia).cuda()
    xd = torch.zeros_like(bd)
    dev = dda.solve_batch("qmrccg", bd, xd, ad, maxit=300, tol=TOL)
    np.testing.assert_array_equal(dev.itno, host.itno)
    np.testing.assert_array_equal(dev.status, host.status)
    assert np.allclose(xd.cpu().numpy(), xh, rtol=0, atol=1e-6 * np.abs(xh).max())
    dda.release()


@pytest.mark.gpu
def test_residual_f64_matches_oracle():
    n = 12
    prob = targets.make_problem(n, m=1.5 + 0.01j, x=2.0)
    rng = np.random.default_rng(5)
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    x = (rng.normal(size=b.shape) + 1j * rng.normal(size=b.shape)).astype(np.complex64) * 0.1
    x[:, np.tile(prob.iocc == 0, 3)] = 0
    aoff = (0.05 * (rng.normal(size=b.shape) + 1j * rng.normal(size=b.shape))).astype(np.complex64)
    got = dda.residual_f64(b, x, adia, aoff)
    gp = O.GreenParams(n, n, n, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    for r in range(b.shape[0]):
        y = op.apply_full(x[r], adia[r], aoff[r])
        occ = op.occ
        bc = O.gather_compact(b[r], occ, op.nat).astype(np.complex128)  # float64 norms
        yc = O.gather_compact(y, occ, op.nat)
        ref = np.linalg.norm(bc - yc) / np.linalg.norm(bc)
        assert abs(got[r] - ref) <= 1e-9 * ref
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["qmrccg", "pbcgs2"])
def test_batch_residual_replacement(name):
    """Residual replacement instead of restarts (DDSCAT_B200_REPLACE_RESIDUAL):
    every RHS still converges on its true residual, passes the FP64 check and
    agrees with the restart-policy solution."""
    n = 24
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=6.0, orientations=targets.random_orientations(3, seed=7))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    xr, xp = np.zeros_like(b), np.zeros_like(b)
    rest = dda.solve_batch(name, b, xr, adia, maxit=2000, tol=TOL)
    rep = dda.solve_batch(name, b, xp, adia, maxit=2000, tol=TOL, replace=True)
    assert np.all(rep.status == 0) and np.all(rep.tole <= TOL)
    assert np.all(dda.residual_f64(b, xp, adia) <= 1.2 * TOL)
    for r in range(b.shape[0]):
        assert np.linalg.norm(xp[r] - xr[r]) / np.linalg.norm(xr[r]) < 20 * TOL
    assert rest.itno.sum() > 0 and rep.itno.sum() > 0
    dda.release()


@pytest.mark.gpu
def test_batch_qmrccg_symmetric_form():
    """One-MATVEC QMRCCG (DDSCAT_B200_QMR_SYMMETRIC): same iterates as the
    two-product form up to rounding, half the MATVECs per iteration."""
    n = 24
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=6.0, orientations=targets.random_orientations(3, seed=9))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    for replace in (False, True):
        x2, x1 = np.zeros_like(b), np.zeros_like(b)
        two = dda.solve_batch("qmrccg", b, x2, adia, maxit=2000, tol=TOL, replace=replace)
        one = dda.solve_batch("qmrccg", b, x1, adia, maxit=2000, tol=TOL, replace=replace, symmetric=True)
        assert np.all(one.status == 0) and np.all(one.tole <= TOL)
        assert np.all(dda.residual_f64(b, x1, adia) <= 1.2 * TOL)
        for r in range(b.shape[0]):
            assert np.linalg.norm(x1[r] - x2[r]) / np.linalg.norm(x2[r]) < 20 * TOL
            # 1 MATVEC per iteration + init + checks, against 2 per iteration
            assert one.ncompte[r] <= 0.6 * two.ncompte[r] * one.itno[r] / max(two.itno[r], 1) + 20
    with pytest.raises(D.DDSCATError):
        dda.solve_batch("pbcgs2", b, np.zeros_like(b), adia, maxit=10, tol=TOL, symmetric=True)
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 24])
def test_batch_qmrccg_graph_matches_host_driven(n):
    """Device-driven iterations in a CUDA graph (DDSCAT_B200_GRAPH) follow the
    host-driven one-MATVEC QMRCCG with residual replacement: iteration counts
    within one, solutions within 20*TOL, FP64 residual <= 1.2*TOL."""
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=5.0, orientations=targets.random_orientations(4, seed=12))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    xh, xg = np.zeros_like(b), np.zeros_like(b)
    host = dda.solve_batch("qmrccg", b, xh, adia, maxit=2000, tol=TOL, replace=True, symmetric=True)
    l0 = dda.launch_count()
    gr = dda.solve_batch("qmrccg", b, xg, adia, maxit=2000, tol=TOL, replace=True, symmetric=True, graph=True)
    assert dda.launch_count() > l0
    assert np.all(gr.status == 0) and np.all(gr.tole <= TOL)
    assert np.all(np.abs(gr.itno - host.itno) <= 1), (gr.itno, host.itno)
    assert np.all(np.abs(gr.ncompte - host.ncompte) <= 2)
    assert np.all(dda.residual_f64(b, xg, adia) <= 1.2 * TOL)
    for r in range(b.shape[0]):
        assert np.linalg.norm(xg[r] - xh[r]) / np.linalg.norm(xh[r]) < 20 * TOL
    ms, rhs, calls = dda.last_solve_stats()
    assert rhs == int(gr.ncompte.sum()) and ms > 0
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 24])
def test_batch_pbcgs2_graph_matches_host_driven(n):
    """Device-driven PBCGS2 iterations (DDSCAT_B200_GRAPH with residual
    replacement: FP64 scalars and the 3 x 3 minimal-residual step in
    single-thread kernels, the reliable-residual check and the reliable update
    in IF conditional nodes) follow the host-driven batched PBCGS2: iteration
    counts within one, solutions within 20*TOL, FP64 residual <= 1.2*TOL."""
    prob = targets.make_problem(n, m=1.5 + 0.02j, x=5.0, orientations=targets.random_orientations(3, seed=7))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    xh, xg = np.zeros_like(b), np.zeros_like(b)
    host = dda.solve_batch("pbcgs2", b, xh, adia, maxit=2000, tol=TOL, replace=True)
    l0 = dda.launch_count()
    gr = dda.solve_batch("pbcgs2", b, xg, adia, maxit=2000, tol=TOL, replace=True, graph=True)
    assert dda.launch_count() > l0
    assert np.all(gr.status == 0) and np.all(gr.tole <= TOL), (gr.status, gr.tole)
    assert np.all(np.abs(gr.itno - host.itno) <= 1), (gr.itno, host.itno)
    assert np.all(np.abs(gr.ncompte - host.ncompte) <= 6), (gr.ncompte, host.ncompte)
    assert np.all(dda.residual_f64(b, xg, adia) <= 1.2 * TOL)
    for r in range(b.shape[0]):
        assert np.linalg.norm(xg[r] - xh[r]) / np.linalg.norm(xh[r]) < 20 * TOL
    ms, rhs, calls = dda.last_solve_stats()
    assert rhs == int(gr.ncompte.sum()) and ms > 0
    dda.release()


@pytest.mark.gpu
def test_batch_qmrccg_nonzero_initial_guess():
    """A nonzero x0 enters through A x0 (formed only for the RHS whose x0 is
    nonzero; for x0 = 0 the product is exactly zero and is skipped, still
    counted in NCOMPTE): warm-started RHS converge in fewer iterations to the
    same FP64-checked tolerance, zero-started ones as before."""
    n = 16
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=3.0, orientations=targets.random_orientations(2, seed=21))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    x = np.zeros_like(b)
    first = dda.solve_batch("qmrccg", b, x, adia, maxit=500, tol=TOL, replace=True, symmetric=True, graph=True)
    assert np.all(first.status == 0)
    assert np.all(first.ncompte >= first.itno + 1)
    x2 = np.zeros_like(b)
    x2[0] = x[0] * (1.0 + 1e-3)  # warm start for RHS 0 only
    x2[2] = x[2] * (1.0 - 1e-3)
    second = dda.solve_batch("qmrccg", b, x2, adia, maxit=500, tol=TOL, replace=True, symmetric=True, graph=True)
    assert np.all(second.status == 0) and np.all(second.tole <= TOL)
    assert np.all(dda.residual_f64(b, x2, adia) <= 1.2 * TOL)
    assert second.itno[0] < first.itno[0] and second.itno[2] < first.itno[2]
    assert abs(int(second.itno[1]) - int(first.itno[1])) <= 1
    ms, rhs, calls = dda.last_solve_stats()
    assert rhs == int(second.ncompte.sum())
    dda.release()


@pytest.mark.gpu
def test_batch_qmrccg_graph_fused_xy_passes(monkeypatch):
    """The graph-driven QMRCCG on the fused xy passes (DDSCAT_B200_FUSEXY=1,
    32^3: M_x = M_y = 64), whose inverse pass also forms the fused vt^T A vt
    sum over its four-CTA clusters: same iteration counts within one and
    solutions within 20*TOL of the five-pass schedule, FP64 residual <= 1.2*TOL."""
    n = 32
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=5.0, orientations=targets.random_orientations(2, seed=5))
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    b, adia = _batch_inputs(prob)
    x5, xf = np.zeros_like(b), np.zeros_like(b)
    r5 = dda.solve_batch("qmrccg", b, x5, adia, maxit=2000, tol=TOL, replace=True, symmetric=True, graph=True)
    monkeypatch.setenv("DDSCAT_B200_FUSEXY", "1")
    rf = dda.solve_batch("qmrccg", b, xf, adia, maxit=2000, tol=TOL, replace=True, symmetric=True, graph=True)
    assert np.all(rf.status == 0) and np.all(rf.tole <= TOL)
    assert np.all(np.abs(rf.itno - r5.itno) <= 1), (rf.itno, r5.itno)
    assert np.all(dda.residual_f64(b, xf, adia) <= 1.2 * TOL)
    for r in range(b.shape[0]):
        assert np.linalg.norm(xf[r] - x5[r]) / np.linalg.norm(x5[r]) < 20 * TOL
    dda.release()
