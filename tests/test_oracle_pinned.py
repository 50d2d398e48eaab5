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


# ---- configuration-size fixtures (reference_fixtures_c1.npz): the small-sphere
# workload and a 64^3 MATVEC, inputs regenerated from seeds by the fixture script
FIX_C1 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_c1.npz")


def _gen():
    import importlib.util

    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "make_reference_fixtures.py")
    spec = importlib.util.spec_from_file_location("make_reference_fixtures", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def fc1():
    if not os.path.exists(FIX_C1):
        pytest.skip("configuration-size reference fixtures not generated")
    return dict(np.load(FIX_C1))


def test_oracle_matvec64_matches_reference(fc1):
    """64^3 MATVEC, 'N' and 'C': the seeded samples, the norm and the random
    projections of the reference's output (2e-5, complex FP32 reference)."""
    G = _gen()
    dims, iocc, ak, x, adia, aoff, idx, proj = G.mv64_inputs()
    op = O.Operator.from_params(O.GreenParams(*dims, ak=tuple(float(v) for v in ak)), iocc)
    for cw in "NC":
        y = op.apply_full(x, adia, aoff, cw)
        smp, nrm, prj = G.mv64_summary(y, idx, proj)
        assert _rel(smp, fc1[f"M64_{cw}_samples"]) < 2e-5
        assert abs(nrm[0] - fc1[f"M64_{cw}_norm"][0]) <= 2e-5 * nrm[0]
        assert np.abs(prj - fc1[f"M64_{cw}_proj"]).max() <= 2e-5 * nrm[0]


def test_oracle_c1_matches_reference(fc1):
    """The small-sphere workload solved by the reference (PBCGS2, both
    polarisations): its solutions have FP64 true residuals <= 1.2 tol under
    the oracle's operator, and the oracle's EVALQ (1e-6) and SCAT (2e-5:
    Csca, g, f1/f2 on 362 directions) of those solutions equal the
    reference's."""
    G = _gen()
    prob = G.c1_problem()
    k = prob.incid[0].k
    op = O.Operator.from_params(O.GreenParams(32, 32, 32, ak=tuple(float(np.float32(a)) for a in k)), prob.iocc)
    occ = op.occ
    for r in range(2):
        b, adia = prob.rhs(r), prob.adia(r)
        assert np.allclose(fc1[f"C1_{r}_inputs"], [b.astype(np.complex128).sum(), adia.astype(np.complex128).sum()],
                           rtol=1e-12), "the fixture was made from other inputs"
        bc = O.gather_compact(b, occ, prob.nat).astype(np.complex128)
        ac = O.gather_compact(adia, occ, prob.nat).astype(np.complex128)
        oc = np.zeros_like(ac)
        xr = fc1[f"C1_{r}_x"].astype(np.complex128)
        it_ref, tole_ref, nc_ref = fc1[f"C1_{r}_meta"]
        assert tole_ref <= G.C1_TOL
        assert np.linalg.norm(bc - op.apply_compact(xr, ac, oc)) / np.linalg.norm(bc) <= 1.2 * G.C1_TOL
        for g, w in zip(O.evalq(bc, xr, ac, oc, k, 1.0), fc1[f"C1_{r}_evalq"]):
            assert abs(g - w) <= 1e-6 * abs(w)
        aks, em1, em2 = G.c1_directions(prob, r)
        sc = O.scat(xr, occ, 32, 32, 0, k, aks, (1, 1, 1), em1, em2, 1.0, G.C1_ETASCA, prob.incid[r].e, prob.x0)
        cb, cs, g0, g1, g2, cg2, navg = fc1[f"C1_{r}_scat"]
        assert sc["navg"] == int(navg)
        assert sc["csca"] == pytest.approx(cs, rel=2e-5)
        assert abs(sc["cscag"][0] / sc["csca"] - g0 / cs) <= 2e-5
        fmax = max(np.abs(fc1[f"C1_{r}_f1"]).max(), np.abs(fc1[f"C1_{r}_f2"]).max())
        assert np.abs(sc["f1"] - fc1[f"C1_{r}_f1"]).max() <= 2e-5 * fmax
        assert np.abs(sc["f2"] - fc1[f"C1_{r}_f2"]).max() <= 2e-5 * fmax


# ---- edge cases (reference_fixtures_edge.npz; inputs from tests/golden/edge_cases.py)
FIX_EDGE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_edge.npz")


@pytest.fixture(scope="module")
def fedge():
    return dict(np.load(FIX_EDGE))


def _edge_cases():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import edge_cases
    return edge_cases


@pytest.mark.parametrize("name", ["pbcgs2", "qmrccg", "pbcgst", "petrkp", "gpbicg"])
def test_oracle_solvers_with_cxaoff_match_reference(fedge, name):
    """Anisotropic sites (nonzero CXAOFF): the oracle's solution of each solver
    equals the reference's within 20*TOL, from the same recurrence."""
    EC = _edge_cases()
    prob, b, adia, aoff = EC.aoff_problem()
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    c = lambda v: O.gather_compact(v, op.occ, prob.nat).astype(np.complex128)  # noqa: E731
    bc, ac, oc = c(b), c(adia), c(aoff)
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    mvh = lambda v: op.apply_compact(v, ac, oc, "C")  # noqa: E731
    x0 = np.zeros_like(bc)
    if name == "pbcgst":
        res = O.solve_pbcgst(mv, bc, x0, EC.MAXIT, EC.TOL, ac)
    elif name == "petrkp":
        res = O.solve_petrkp(mv, mvh, bc, x0, EC.MAXIT, EC.TOL)
    else:
        res = O.SOLVERS[name](mv, bc, x0, EC.MAXIT, EC.TOL)
    assert res.status == int(fedge[f"O_{name}_rc"][0]) == 0
    ref = c(fedge[f"O_{name}_x"])
    assert np.linalg.norm(res.x - ref) / np.linalg.norm(ref) < 20 * EC.TOL


@pytest.mark.parametrize("case", ["single_site", "hollow16", "hollow18x12x10"])
def test_oracle_sparse_matvec_matches_reference(fedge, case):
    EC = _edge_cases()
    prob, b, adia, aoff, x = EC.sparse_problem(case)
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    for cw in "NC":
        y = op.apply_full(x, adia, aoff, cw)
        ref = fedge[f"S_{case}_y{cw}"]
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 2e-5


# ---- periodic targets (reference_fixtures_pbc.npz, IPBC = 1): replica-sum Green
# tensor and full-tensor MATVEC for periodicity in y, z and y+z, with IDIPINT 0
# and 1, and a PBCGS2 solve with EVALQ and SCAT amplitudes on a slab periodic in
# y and z; inputs regenerated by tests/golden/edge_cases.py
FIX_PBC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_pbc.npz")


@pytest.fixture(scope="module")
def fpbc():
    return dict(np.load(FIX_PBC))


def _pbc_operator(cs):
    gp = O.GreenParams(*cs["dims"], ipbc=1, idipint=cs["idipint"], gamma=cs["gamma"], pyd=cs["pyd"], pzd=cs["pzd"],
                       ak=tuple(float(a) for a in cs["ak"]))
    return O.Operator.from_params(gp, cs["iocc"])


@pytest.mark.parametrize("case", ["y", "z", "yz", "yf"])
def test_oracle_periodic_matvec_matches_reference(fpbc, case):
    cs = {c["name"]: c for c in _edge_cases().pbc_cases()}[case]
    op = _pbc_operator(cs)
    for cw in "NC":
        y = op.apply_full(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fpbc[f"M_{case}_y{cw}"]) < 2e-5


def test_oracle_periodic_solve_matches_reference(fpbc):
    EC = _edge_cases()
    prob, gamma, pyd, pzd, aks, em1, em2 = EC.pbc_solve_problem()
    k = prob.incid[0].k.astype(np.float32).astype(np.float64)
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ipbc=1, gamma=gamma, pyd=pyd, pzd=pzd, ak=tuple(k))
    op = O.Operator.from_params(gp, prob.iocc)
    occ = op.occ
    c = lambda v: O.gather_compact(v, occ, prob.nat).astype(np.complex128)  # noqa: E731
    bc, ac, oc = c(prob.rhs(0)), c(prob.adia(0)), c(prob.aoff())
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    it_ref, tole_ref, nc_ref = fpbc["P_meta"]
    assert int(fpbc["P_rc"][0]) == 0 and tole_ref <= TOL
    res = O.solve_pbcgs2(mv, bc, np.zeros_like(bc), 300, TOL)
    assert res.status == 0 and abs(res.itno - it_ref) <= 1 and abs(res.ncompte - nc_ref) <= 2
    xr = c(fpbc["P_x"])
    assert np.linalg.norm(res.x - xr) / np.linalg.norm(xr) < 20 * TOL
    for g, r in zip(O.evalq(bc, xr, ac, oc, k, 1.0), fpbc["P_evalq"]):
        assert abs(g - r) <= 1e-6 * abs(r)
    # JPBC = 3: SCAT skips the finite-target integration (zero sums, NAVG = 0)
    # and returns the amplitudes in the selected directions
    sc = O.scat(xr, occ, prob.nx, prob.ny, 3, k, aks, (1, 1, 1), em1, em2, 1.0, 0.0, None, prob.x0)
    assert sc["navg"] == 0 and np.all(fpbc["P_scat"] == 0)
    fmax = np.abs(fpbc["P_f1"]).max()
    assert np.abs(sc["f1"] - fpbc["P_f1"]).max() <= 2e-5 * fmax
    assert np.abs(sc["f2"] - fpbc["P_f2"]).max() <= 2e-5 * fmax


def test_oracle_periodic_cpu_green_matvec_matches_reference(fpbc):
    """prepare_f32 with IPBC = 1: the full-tensor MATVEC on a caller-supplied
    planar (6, 2nz, 2ny, 2nx) spectrum."""
    cs = _edge_cases().pbc_cpu_green_case()
    op = O.Operator(*cs["dims"], cs["green"].astype(np.complex128), cs["iocc"])
    for cw in "NC":
        y = op.apply_full(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fpbc[f"M_cpu_y{cw}"]) < 2e-5


# ---- rectangular lattices (reference_fixtures_dx.npz): dx1..dx3 = 1.0, 0.9, 1.1
FIX_DX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_dx.npz")


@pytest.fixture(scope="module")
def fdx():
    return dict(np.load(FIX_DX))


@pytest.mark.parametrize("case", ["iso", "flt", "pbc"])
def test_oracle_rectangular_lattice_matvec_matches_reference(fdx, case):
    EC = _edge_cases()
    cs = {c["name"]: c for c in EC.dx_cases()}[case]
    gp = O.GreenParams(*cs["dims"], ipbc=cs["ipbc"], idipint=cs["idipint"], gamma=cs["gamma"], pyd=cs["pyd"],
                       pzd=0.0, dx=EC.DX, ak=tuple(float(a) for a in cs["ak"]))
    op = O.Operator.from_params(gp, cs["iocc"])
    for cw in "NC":
        y = op.apply_full(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fdx[f"M_{case}_y{cw}"]) < 2e-5


def test_oracle_rectangular_lattice_solve_matches_reference(fdx):
    EC = _edge_cases()
    prob, aks, em1, em2 = EC.dx_solve_problem()
    k = prob.incid[0].k.astype(np.float32).astype(np.float64)
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, dx=EC.DX, ak=tuple(k))
    op = O.Operator.from_params(gp, prob.iocc)
    occ = op.occ
    c = lambda v: O.gather_compact(v, occ, prob.nat).astype(np.complex128)  # noqa: E731
    bc, ac, oc = c(prob.rhs(0)), c(prob.adia(0)), c(prob.aoff())
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    it_ref, tole_ref, nc_ref = fdx["Q_meta"]
    assert int(fdx["Q_rc"][0]) == 0 and tole_ref <= TOL
    res = O.SOLVERS["qmrccg"](mv, bc, np.zeros_like(bc), 300, TOL)
    assert res.status == 0 and abs(res.itno - it_ref) <= 1 and abs(res.ncompte - nc_ref) <= 2
    xr = c(fdx["Q_x"])
    assert np.linalg.norm(res.x - xr) / np.linalg.norm(xr) < 20 * TOL
    for g, r in zip(O.evalq(bc, xr, ac, oc, k, 1.0), fdx["Q_evalq"]):
        assert abs(g - r) <= 1e-6 * abs(r)
    sc = O.scat(xr, occ, prob.nx, prob.ny, 0, k, aks, EC.DX, em1, em2, 1.0, 3.0, prob.incid[0].e, prob.x0)
    cb, cs, g0, g1, g2, cg2, navg = fdx["Q_scat"]
    assert sc["navg"] == int(navg)
    assert sc["csca"] == pytest.approx(cs, rel=2e-5)
    assert sc["cscag2"] == pytest.approx(cg2, rel=2e-5)
    for a, r in zip(sc["cscag"], (g0, g1, g2)):
        assert abs(a - r) <= 2e-5 * cs
    assert abs(sc["cbksca"] - cb) <= 2e-5 * cs
    fmax = np.abs(fdx["Q_f1"]).max()
    assert np.abs(sc["f1"] - fdx["Q_f1"]).max() <= 2e-5 * fmax
    assert np.abs(sc["f2"] - fdx["Q_f2"]).max() <= 2e-5 * fmax


# ---- limit cases of all eight solvers (reference_fixtures_limits.npz): MAXIT
# reached, a zero right-hand side, a nonzero initial guess
FIX_LIM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_limits.npz")
LIMIT_CASES = (("maxit", 3, 1e-12), ("zero", 10, 1e-5), ("x0", 300, 1e-5))


@pytest.fixture(scope="module")
def flim():
    return dict(np.load(FIX_LIM))


@pytest.fixture(scope="module")
def lim_operator():
    prob, b, adia, aoff, x0 = _edge_cases().limits_problem()
    gp = O.GreenParams(prob.nx, prob.ny, prob.nz, ak=tuple(float(np.float32(a)) for a in prob.incid[0].k))
    op = O.Operator.from_params(gp, prob.iocc)
    c = lambda v: O.gather_compact(v, op.occ, prob.nat).astype(np.complex128)  # noqa: E731
    return op, c(b), c(adia), c(aoff), c(x0), c


@pytest.mark.parametrize("name", SOLVER_NAMES)
def test_oracle_solver_limits_match_reference(flim, lim_operator, name):
    """Return code and ITNO in every case (the reference's codes for a zero
    right-hand side: GPBICG 32, QMRCCG 52, PBCGST 78, PETRKP 115, BiCGStab(4)
    133, GPBiCGStab(2) 153, GPBiCGStab(4) 183, PBCGS2 0 with TOLE = inf; MAXIT
    reached: PBCGST 87, the others 0); NCOMPTE and the iterate where the solve
    returns 0."""
    op, bc, ac, oc, x0c, c = lim_operator
    mv = lambda v: op.apply_compact(v, ac, oc)  # noqa: E731
    mvh = lambda v: op.apply_compact(v, ac, oc, "C")  # noqa: E731
    for tag, maxit, tol in LIMIT_CASES:
        b = np.zeros_like(bc) if tag == "zero" else bc
        x0 = x0c.copy() if tag == "x0" else np.zeros_like(bc)
        if name == "pbcgst":
            res = O.solve_pbcgst(mv, b, x0, maxit, tol, ac)
        elif name == "petrkp":
            res = O.solve_petrkp(mv, mvh, b, x0, maxit, tol)
        else:
            res = O.SOLVERS[name](mv, b, x0, maxit, tol)
        rc = int(flim[f"L_{name}_{tag}_rc"][0])
        it_ref, tole_ref, nc_ref = flim[f"L_{name}_{tag}_meta"]
        assert res.status == rc and res.itno == int(it_ref), (tag, res.status, rc, res.itno, it_ref)
        if rc == 0:
            assert res.ncompte == int(nc_ref), (tag, res.ncompte, nc_ref)
            xr = c(flim[f"L_{name}_{tag}_x"])
            if np.linalg.norm(xr) > 0:
                assert np.linalg.norm(res.x - xr) / np.linalg.norm(xr) < 2 * TOL, tag
