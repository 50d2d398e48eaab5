"""Edge cases of the drop-in path, against the FP64 oracle and against the
reference library's own outputs on the same inputs
(tests/golden/reference_fixtures_edge.npz, written on a B200 by
tests/golden/make_reference_fixtures.py from the unmodified reference).

* Anisotropic sites (nonzero CXAOFF) through the single-RHS solvers: the
  solver calls gather CXADIA and CXAOFF into the compact layout of the Krylov
  vectors, and PBCGST's DIAGL preconditioner reads CXADIA in the full layout.
  The off-diagonal blocks are symmetric per site, so the matrix stays complex
  symmetric (QMRCCG's assumption, cu:1090).
* A target of one occupied site, and hollow targets (a shell with two
  separated blobs and vacant planes) whose x rows, y columns and z planes are
  partly or wholly vacant, for the compact gather/scatter of the first and last
  MATVEC passes.
Bars: the reference's return code; for converged solves TOLE <= TOL, the FP64
true residual <= 1.2*TOL and the solution within 20*TOL of the reference's;
MATVEC relative L2 error <= 2e-5 against the oracle and the reference, vacant
sites exactly 0.  On the single isolated site the system is diagonal and the
first BiCG step solves it exactly: in FP32 the next Lanczos vector is exactly
zero, and the reference's recurrences stop with their breakdown codes (PBCGS2
98 on SIGMA = 0, QMRCCG 58 on GAMMA = 0) before the solution update; the same
codes are required here.
"""
import os
import sys

import numpy as np
import pytest

import ddscat_b200 as D
from oracle import ddscat_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import edge_cases as EC  # noqa: E402

FIX = os.path.join(HERE, "golden", "reference_fixtures_edge.npz")


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(FIX))


def _operator(prob):
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    return O.Operator.from_params(gp, prob.iocc)


def _true_residual(op, prob, x, b, adia, aoff):
    c = lambda v: O.gather_compact(v, op.occ, prob.nat).astype(np.complex128)  # noqa: E731
    bc = c(b)
    return np.linalg.norm(bc - op.apply_compact(c(x), c(adia), c(aoff))) / np.linalg.norm(bc)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.gpu
@pytest.mark.parametrize("name", EC.SOLVERS_AOFF)
def test_solvers_with_nonzero_cxaoff(fx, name):
    prob, b, adia, aoff = EC.aoff_problem()
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k)
    out = dda.solve(name, b, adia, aoff, maxit=EC.MAXIT, tol=EC.TOL)
    assert out.rc == int(fx[f"O_{name}_rc"][0]) == 0 and out.tole <= EC.TOL
    op = _operator(prob)
    assert _true_residual(op, prob, out.x, b, adia, aoff) <= 1.2 * EC.TOL
    assert _rel(out.x, fx[f"O_{name}_x"]) < 20 * EC.TOL
    ref_it = fx[f"O_{name}_meta"][0]
    assert abs(out.itno - ref_it) <= max(3, 0.2 * ref_it)
    assert np.all(out.x.reshape(3, -1)[:, prob.iocc == 0] == 0)
    # the same operator through the MATVEC entry point
    y = dda.apply(out.x, adia, aoff)
    assert _rel(y, op.apply_full(out.x, adia, aoff)) <= 2e-5
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ("single_site",) + EC.HOLLOW)
def test_sparse_targets(fx, case):
    prob, b, adia, aoff, x = EC.sparse_problem(case)
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k)
    op = _operator(prob)
    for cw in ("N", "C"):
        y = dda.apply(x, adia, aoff, cw)
        assert _rel(y, op.apply_full(x, adia, aoff, cw)) <= 2e-5
        assert _rel(y, fx[f"S_{case}_y{cw}"]) <= 2e-5
        assert np.all(y.reshape(3, -1)[:, prob.iocc == 0] == 0)
    for name in ("pbcgs2", "qmrccg"):
        out = dda.solve(name, b, adia, aoff, maxit=400, tol=EC.TOL, check=False)
        assert out.rc == int(fx[f"S_{case}_{name}_rc"][0]), (name, out.rc)
        if out.rc == 0:
            assert out.tole <= EC.TOL
            assert _true_residual(op, prob, out.x, b, adia, aoff) <= 1.2 * EC.TOL
    dda.release()
