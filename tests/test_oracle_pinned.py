"""Pins the CPU oracle to the reference implementation: the fixtures in
tests/golden/reference_fixtures.npz were produced by the unmodified reference
library (ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu built by oracle/Makefile)
running on a B200 (tests/golden/make_reference_fixtures.py).  CPU only.

Tolerances: MATVEC 2e-5 relative L2 (the reference computes in complex FP32);
EVALQ 1e-6; SCAT 2e-5 (the reference evaluates phases with FP32 sincosf)."""
import os

import numpy as np
import pytest

from oracle import ddscat_oracle as O

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures.npz")
TOL = 1e-5


@pytest.fixture(scope="module")
def fx():
    return dict(np.load(FIX))


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.mark.parametrize("idip", [0, 1])
def test_oracle_matvec_matches_reference(fx, idip):
    nx, ny, nz = (int(v) for v in fx[f"A{idip}_dims"])
    gp = O.GreenParams(nx, ny, nz, idipint=idip, ak=tuple(float(v) for v in fx[f"A{idip}_ak"]))
    op = O.Operator.from_params(gp, fx[f"A{idip}_iocc"])
    for cw in "NC":
        y = op.apply_full(fx[f"A{idip}_x"], fx[f"A{idip}_adia"], fx[f"A{idip}_aoff"], cw)
        assert _rel(y, fx[f"A{idip}_y{cw}"]) < 2e-5


def test_oracle_matvec_with_cpu_green_matches_reference(fx):
    nx, ny, nz = (int(v) for v in fx["C_dims"])
    nat = nx * ny * nz
    op = O.Operator.from_octant(nx, ny, nz, fx["C_oct"].astype(np.complex128), np.ones(nat, dtype=np.int16))
    y = op.apply_full(fx["C_x"], fx["C_adia"], np.zeros(3 * nat))
    assert _rel(y, fx["C_y"]) < 2e-5


def _b_operator(fx):
    n = int(fx["B_n"][0])
    gp = O.GreenParams(n, n, n, ak=tuple(float(v) for v in fx["B_k"]))
    op = O.Operator.from_params(gp, fx["B_iocc"])
    occ = op.occ
    bc = O.gather_compact(fx["B_b"], occ, op.nat).astype(np.complex128)
    ac = O.gather_compact(fx["B_adia"], occ, op.nat).astype(np.complex128)
    oc = np.zeros_like(ac)
    return op, occ, bc, ac, oc


SOLVER_NAMES = ["gpbicg", "qmrccg", "pbcgst", "pbcgs2", "petrkp", "bicgstab4", "gpbicgstab2", "gpbicgstab4"]


@pytest.mark.parametrize("name", SOLVER_NAMES)
def test_oracle_solver_matches_reference(fx, name):
    op, occ, bc, ac, oc = _b_operator(fx)
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    mvh = lambda v: op.apply_compact(v, ac, oc, "C")  # noqa: E731
    assert int(fx[f"B_{name}_rc"][0]) == 0
    it_ref, tole_ref, nc_ref = fx[f"B_{name}_meta"]
    xr = O.gather_compact(fx[f"B_{name}_x"], occ, op.nat).astype(np.complex128)
    true = np.linalg.norm(bc - mv(xr)) / np.linalg.norm(bc)
    assert true <= 1.2 * TOL
    assert tole_ref <= TOL
    x0 = np.zeros_like(bc)
    if name == "pbcgst":
        res = O.solve_pbcgst(mv, bc, x0, 300, TOL, ac)
    elif name == "petrkp":
        res = O.solve_petrkp(mv, mvh, bc, x0, 300, TOL)
    else:
        res = O.SOLVERS[name](mv, bc, x0, 300, TOL)
    # same algorithm: the iteration and MATVEC counts agree with the reference's
    assert abs(res.itno - it_ref) <= max(1, 0.2 * it_ref), (res.itno, it_ref)
    assert abs(res.ncompte - nc_ref) <= max(2, 0.2 * nc_ref), (res.ncompte, nc_ref)
    assert np.linalg.norm(res.x - xr) / np.linalg.norm(xr) < 20 * TOL


def test_oracle_evalq_and_scat_match_reference(fx):
    op, occ, bc, ac, oc = _b_operator(fx)
    k = fx["B_k"].astype(np.float64)
    xr = O.gather_compact(fx["B_qmrccg_x"], occ, op.nat)
    got = O.evalq(bc, xr, ac, oc, k, 1.0)
    for g, r in zip(got, fx["B_evalq"]):
        assert abs(g - r) <= 1e-6 * abs(r)
    n = int(fx["B_n"][0])
    sc = O.scat(xr, occ, n, n, 0, k, fx["B_aks"], (1, 1, 1), fx["B_em1"], fx["B_em2"], 1.0, 3.0, fx["B_e"],
                fx["B_x0"])
    cb, cs, g0, g1, g2, cg2, navg = fx["B_scat"]
    assert sc["navg"] == int(navg)
    assert sc["csca"] == pytest.approx(cs, rel=2e-5)
    assert sc["cscag2"] == pytest.approx(cg2, rel=2e-5)
    for a, r in zip(sc["cscag"], (g0, g1, g2)):
        assert abs(a - r) <= 2e-5 * cs
    assert abs(sc["cbksca"] - cb) <= 2e-5 * cs
    fmax = np.abs(fx["B_f1"]).max()
    assert np.abs(sc["f1"] - fx["B_f1"]).max() <= 2e-5 * fmax
    assert np.abs(sc["f2"] - fx["B_f2"]).max() <= 2e-5 * fmax
