"""All-FP64 batched solve (ddscat_b200_solve_batch_f64) and the Q error of the
FP32 batched solve against it.

* The FP64 solution meets a 1e-10 tolerance on the FP64 oracle operator
  (relative true residual <= 1e-9).
* Cext and Cabs from the FP32 solution (tol 1e-5, EVALQ on the GPU) agree with
  those of the FP64 solution to <= 1e-4 relative, the bar the batched FP32
  path is held to."""
import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets
from oracle import ddscat_oracle as O


@pytest.mark.gpu
@pytest.mark.parametrize("name,symmetric", [("qmrccg", True), ("pbcgs2", False)])
def test_fp64_batch_solve_and_q_errors(name, symmetric):
    n = 16
    prob = targets.make_problem(n, m=1.33 + 0.05j, x=3.0, orientations=targets.random_orientations(2, seed=5))
    R = len(prob.incid)
    b = np.stack([prob.rhs(r) for r in range(R)])
    adia = np.stack([prob.adia(r) for r in range(R)])
    dda = D.DDA()
    dda.prepare_green(n, n, n, prob.iocc, prob.incid[0].k)
    x64 = np.zeros(b.shape, dtype=np.complex128)
    out64 = dda.solve_batch_f64(name, b, x64, adia, maxit=2000, tol=1e-10, replace=True, symmetric=symmetric)
    assert np.all(out64.status == 0) and np.all(out64.tole <= 1e-10)
    gp = O.GreenParams(n, n, n, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    aoff = np.zeros(b.shape[1], dtype=np.complex128)
    occ = prob.occ
    for r in range(R):
        y = op.apply_full(x64[r], adia[r].astype(np.complex128), aoff)
        bc = O.gather_compact(b[r].astype(np.complex128), occ, prob.nat)
        yc = O.gather_compact(y, occ, prob.nat)
        assert np.linalg.norm(bc - yc) / np.linalg.norm(bc) <= 1e-9
    x32 = np.zeros_like(b)
    out32 = dda.solve_batch(name, b, x32, adia, maxit=2000, tol=1e-5, replace=True, symmetric=symmetric)
    assert np.all(out32.status == 0)
    for r in range(R):
        k = prob.incid[r].k
        ec, ac = O.gather_compact(b[r], occ, prob.nat), O.gather_compact(adia[r], occ, prob.nat)
        oc = np.zeros_like(ac)
        q32 = dda.evalq(k, use_resident=0, e=ec, p=O.gather_compact(x32[r], occ, prob.nat), adia=ac, aoff=oc)
        q64 = dda.evalq(k, use_resident=0, e=ec, p=O.gather_compact(x64[r], occ, prob.nat).astype(np.complex64),
                        adia=ac, aoff=oc)
        for a, c in zip(q32[:2], q64[:2]):  # Cabs, Cext
            assert abs(a - c) <= 1e-4 * abs(c), (r, a, c)
    dda.release()
