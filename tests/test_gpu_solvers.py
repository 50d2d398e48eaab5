"""GPU parity of the eight Krylov solvers (ddscat_cuda_solve_*_f32) against the
FP64 oracle restatements of the same algorithms.

Checks per solver, on a seeded 12^3 sphere and a 10x8x6 ellipsoid:
  * return code 0 and TOLE <= TOL (the reference's contract);
  * the FP64 true residual of the returned x <= 1.2*TOL (FP32 MATVEC error
    allowance);
  * x agrees with the FP64 direct solve to 20*TOL relative;
  * iteration count within max(3, 30 %) of the FP64 oracle's;
  * NCOMPTE >= the MATVECs the iteration count implies.
"""
import os

import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets
from oracle import ddscat_oracle as O

TOL = 1e-5


def _setup(n=12, dims=None, m=1.5 + 0.01j, x=2.0, semi=None, r=0):
    if dims is None:
        prob = targets.make_problem(n, m=m, x=x)
    else:
        prob = targets.make_problem(dims[0], dims[1], dims[2], m=m, x=x, semi=semi)
    ak = prob.incid[r].k
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(float(np.float32(a)) for a in ak))
    op = O.Operator.from_params(gp, prob.iocc)
    b, adia, aoff = prob.rhs(r), prob.adia(r), prob.aoff()
    occ = op.occ
    bc = O.gather_compact(b, occ, prob.nat).astype(np.complex128)
    ac = O.gather_compact(adia, occ, prob.nat).astype(np.complex128)
    oc = np.zeros_like(ac)
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    mvh = lambda v: op.apply_compact(v, ac, oc, "C")  # noqa: E731
    return prob, op, b, adia, aoff, bc, ac, mv, mvh


def _oracle_solve(name, mv, mvh, bc, ac, maxit=400):
    x0 = np.zeros_like(bc)
    if name == "pbcgst":
        return O.solve_pbcgst(mv, bc, x0, maxit, TOL, ac)
    if name == "petrkp":
        return O.solve_petrkp(mv, mvh, bc, x0, maxit, TOL)
    return O.SOLVERS[name](mv, bc, x0, maxit, TOL)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", ["sphere12", "ellipsoid"])
@pytest.mark.parametrize("name", D.SOLVERS)
def test_solver_parity(name, shape):
    if shape == "sphere12":
        prob, op, b, adia, aoff, bc, ac, mv, mvh = _setup(12)
    else:
        prob, op, b, adia, aoff, bc, ac, mv, mvh = _setup(dims=(10, 8, 6), m=1.33 + 0.05j, x=1.5)
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k)
    out = dda.solve(name, b, adia, aoff, maxit=400, tol=TOL)
    assert out.rc == 0
    assert out.tole <= TOL
    xc = O.gather_compact(out.x, op.occ, prob.nat).astype(np.complex128)
    # unoccupied sites of the returned full vector are zero
    assert np.all(out.x.reshape(3, -1)[:, prob.iocc == 0] == 0)
    true = np.linalg.norm(bc - mv(xc)) / np.linalg.norm(bc)
    assert true <= 1.2 * TOL, true
    ref = _oracle_solve(name, mv, mvh, bc, ac)
    assert ref.status == 0
    xd = O.solve_qmrccg(mv, bc, np.zeros_like(bc), 2000, 1e-12).x
    assert np.linalg.norm(xc - xd) / np.linalg.norm(xd) < 20 * TOL
    assert abs(out.itno - ref.itno) <= max(3, 0.3 * ref.itno), (out.itno, ref.itno)
    assert out.ncompte >= out.itno
    dda.release()


@pytest.mark.gpu
def test_initial_guess_and_maxit_semantics():
    prob, op, b, adia, aoff, bc, ac, mv, mvh = _setup(10)
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k)
    # MAXIT reached: PBCGS2 returns 0 with TOLE > TOL; PBCGST returns 87 but still writes x
    o1 = dda.solve("pbcgs2", b, adia, aoff, maxit=1, tol=1e-12, check=False)
    assert o1.rc == 0 and o1.itno == 1 and o1.tole > 1e-12
    o2 = dda.solve("pbcgst", b, adia, aoff, maxit=2, tol=1e-12, check=False)
    assert o2.rc == 87 and o2.itno == 2 and np.any(o2.x != 0)
    # QMRCCG honours a nonzero initial guess: starting from the solution it stops at once
    sol = dda.solve("qmrccg", b, adia, aoff, maxit=400, tol=TOL)
    again = dda.solve("qmrccg", b, adia, aoff, x0=sol.x, maxit=400, tol=TOL)
    assert again.itno <= 1
    # zero RHS is rejected by QMRCCG with the reference's code 52
    z = dda.solve("qmrccg", np.zeros_like(b), adia, aoff, maxit=10, tol=TOL, check=False)
    assert z.rc == 52
    dda.release()


@pytest.mark.gpu
def test_config_c1_sphere_q_parity():
    """32^3 sphere, m=1.50+0.01i, x=5, PBCGS2 at 1e-5, two polarisations:
    Qext/Qabs within 1e-4 of the FP64 oracle solve (the accuracy bar for Q values)."""
    prob = targets.make_problem(32, m=1.5 + 0.01j, x=5.0)
    dda = D.DDA()
    dda.prepare_green(32, 32, 32, prob.iocc, prob.incid[0].k)
    gp = O.GreenParams(32, 32, 32, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    occ = op.occ
    for r in range(2):
        b, adia, aoff = prob.rhs(r), prob.adia(r), prob.aoff()
        out = dda.solve("pbcgs2", b, adia, aoff, maxit=300, tol=TOL)
        cabs, cext, cpha = dda.evalq(prob.incid[r].k)
        bc = O.gather_compact(b, occ, prob.nat).astype(np.complex128)
        ac = O.gather_compact(adia, occ, prob.nat).astype(np.complex128)
        oc = np.zeros_like(ac)
        mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
        ref = O.solve_pbcgs2(mv, bc, np.zeros_like(bc), 300, 1e-8)
        qa, qe, _ = O.evalq(bc, ref.x, ac, oc, prob.incid[r].k, 1.0)
        assert abs(cext - qe) / abs(qe) < 1e-4
        assert abs(cabs - qa) / abs(qa) < 1e-4
    dda.release()


@pytest.mark.gpu
def test_abi_console_lines_on_by_default(capfd):
    """The reference entry points print the reference's console lines by
    default (one per MATVEC with its GPU time, cu:417, and one per iteration,
    e.g. cu:1085-1092), which DDSCAT users see; level 0 silences them."""
    prob = targets.make_problem(12, m=1.5 + 0.01j, x=2.0)
    dda = D.DDA()
    dda.prepare_green(12, 12, 12, prob.iocc, prob.incid[0].k)
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    try:
        dda.lib.ddscat_b200_set_verbose(-1)  # the default (DDSCAT_B200_VERBOSE unset: on)
        if os.environ.get("DDSCAT_B200_VERBOSE", "1") == "0":
            pytest.skip("DDSCAT_B200_VERBOSE=0 in this environment")
        capfd.readouterr()
        out = dda.solve("qmrccg", b, adia, aoff, maxit=200, tol=1e-5)
        text = capfd.readouterr().out
        assert " QMRCCG iteration=" in text
        assert "CUDA MATVEC" in text and "[N,QMRCCG]: GPU=" in text
        assert text.count("[N,QMRCCG]") == out.ncompte
        dda.apply(b, adia, aoff)
        assert "[N,host-copy]: GPU=" in capfd.readouterr().out
        dda.lib.ddscat_b200_set_verbose(0)
        dda.solve("qmrccg", b, adia, aoff, maxit=200, tol=1e-5)
        assert "CUDA MATVEC" not in capfd.readouterr().out
    finally:
        dda.lib.ddscat_b200_set_verbose(-1)
        dda.release()
