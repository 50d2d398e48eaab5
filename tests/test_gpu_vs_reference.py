"""The B200 library against the reference library's own outputs on identical
inputs (tests/golden/reference_fixtures.npz, produced by the unmodified
reference on a B200).  Tolerances as in test_oracle_pinned.py; solver
iteration counts must agree within 20 % (both are FP32-vector / FP64-scalar
implementations of the same recurrences)."""
import os

import numpy as np
import pytest

import ddscat_b200 as D
from oracle import ddscat_oracle as O

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures.npz")
TOL = 1e-5


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(FIX))


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
@pytest.mark.parametrize("idip", [0, 1])
def test_matvec_vs_reference(fx, idip, layout):
    dims = [int(v) for v in fx[f"A{idip}_dims"]]
    dda = D.DDA(layout)
    dda.prepare_green(*dims, fx[f"A{idip}_iocc"], fx[f"A{idip}_ak"], idipint=idip)
    for cw in "NC":
        y = dda.apply(fx[f"A{idip}_x"], fx[f"A{idip}_adia"], fx[f"A{idip}_aoff"], cw)
        assert _rel(y, fx[f"A{idip}_y{cw}"]) < 2e-5
    dda.release()


@pytest.mark.gpu
def test_prepare_f32_vs_reference(fx):
    dims = [int(v) for v in fx["C_dims"]]
    nat = int(np.prod(dims))
    dda = D.DDA()
    dda.prepare(*dims, np.ones(nat, dtype=np.int16), fx["C_oct"])
    y = dda.apply(fx["C_x"], fx["C_adia"], np.zeros(3 * nat, dtype=np.complex64))
    assert _rel(y, fx["C_y"]) < 2e-5
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("name", D.SOLVERS)
def test_solver_vs_reference(fx, name):
    n = int(fx["B_n"][0])
    dda = D.DDA()
    dda.prepare_green(n, n, n, fx["B_iocc"], fx["B_k"])
    out = dda.solve(name, fx["B_b"], fx["B_adia"], fx["B_aoff"], maxit=300, tol=TOL)
    it_ref, tole_ref, nc_ref = fx[f"B_{name}_meta"]
    assert out.rc == int(fx[f"B_{name}_rc"][0]) == 0
    assert abs(out.itno - it_ref) <= max(1, 0.2 * it_ref), (out.itno, it_ref)
    assert abs(out.ncompte - nc_ref) <= max(2, 0.2 * nc_ref), (out.ncompte, nc_ref)
    assert out.tole <= TOL
    assert _rel(out.x, fx[f"B_{name}_x"]) < 20 * TOL
    if name == "qmrccg":
        k = fx["B_k"]
        got = dda.evalq(k)
        for g, r in zip(got, fx["B_evalq"]):
            assert abs(g - r) <= 1e-4 * abs(r)  # different (converged) iterates
        sc = dda.scat(k, fx["B_e"], fx["B_x0"], etasca=3.0, aks=fx["B_aks"], em1=fx["B_em1"], em2=fx["B_em2"])
        cb, cs, g0, g1, g2, cg2, navg = fx["B_scat"]
        assert sc["navg"] == int(navg)
        assert sc["csca"] == pytest.approx(cs, rel=1e-4)
        fmax = np.abs(fx["B_f1"]).max()
        assert np.abs(sc["f1"] - fx["B_f1"]).max() <= 1e-4 * fmax
    dda.release()
