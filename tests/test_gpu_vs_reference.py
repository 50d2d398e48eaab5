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


# ---- configuration-size fixtures: the small-sphere workload (32^3, PBCGS2,
# EVALQ, SCAT at ETASCA 0.5 on 362 directions) and a 64^3 MATVEC
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


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
def test_matvec64_vs_reference(fc1, layout):
    G = _gen()
    dims, iocc, ak, x, adia, aoff, idx, proj = G.mv64_inputs()
    dda = D.DDA(layout)
    dda.prepare_green(*dims, iocc, ak)
    for cw in "NC":
        y = dda.apply(x, adia, aoff, cw)
        smp, nrm, prj = G.mv64_summary(y, idx, proj)
        assert _rel(smp, fc1[f"M64_{cw}_samples"]) < 2e-5
        assert abs(nrm[0] - fc1[f"M64_{cw}_norm"][0]) <= 2e-5 * nrm[0]
        assert np.abs(prj - fc1[f"M64_{cw}_proj"]).max() <= 2e-5 * nrm[0]
    dda.release()


@pytest.mark.gpu
def test_c1_workload_vs_reference(fc1):
    """This library's ABI on the small-sphere workload against the reference's
    outputs on the same inputs: iteration and MATVEC counts within 20 %,
    solutions within 20 tol, EVALQ's Q and SCAT's Csca within 1e-4 relative,
    g within 1e-4, f1/f2 within 1e-4 of max|f| (two converged FP32 iterates of
    the same recurrence)."""
    G = _gen()
    prob = G.c1_problem()
    k = prob.incid[0].k.astype(np.float32)
    dda = D.DDA()
    dda.prepare_green(32, 32, 32, prob.iocc, k)
    for r in range(2):
        b, adia = prob.rhs(r), prob.adia(r)
        out = dda.solve("pbcgs2", b, adia, prob.aoff(), maxit=G.C1_MAXIT, tol=G.C1_TOL)
        it_ref, tole_ref, nc_ref = fc1[f"C1_{r}_meta"]
        assert out.rc == 0 and out.tole <= G.C1_TOL
        assert abs(out.itno - it_ref) <= max(1, 0.2 * it_ref), (out.itno, it_ref)
        assert abs(out.ncompte - nc_ref) <= max(2, 0.2 * nc_ref), (out.ncompte, nc_ref)
        xc = np.concatenate([out.x[c * prob.nat:(c + 1) * prob.nat][prob.occ] for c in range(3)])
        assert _rel(xc, fc1[f"C1_{r}_x"]) < 20 * G.C1_TOL
        for g, w in zip(dda.evalq(k), fc1[f"C1_{r}_evalq"]):
            assert abs(g - w) <= 1e-4 * abs(w)
        aks, em1, em2 = G.c1_directions(prob, r)
        sc = dda.scat(k, prob.incid[r].e, prob.x0, etasca=G.C1_ETASCA, aks=aks, em1=em1, em2=em2)
        cb, cs, g0, g1, g2, cg2, navg = fc1[f"C1_{r}_scat"]
        assert sc["navg"] == int(navg)
        assert sc["csca"] == pytest.approx(cs, rel=1e-4)
        assert abs(sc["cscag"][0] / sc["csca"] - g0 / cs) <= 1e-4
        fmax = max(np.abs(fc1[f"C1_{r}_f1"]).max(), np.abs(fc1[f"C1_{r}_f2"]).max())
        assert np.abs(sc["f1"] - fc1[f"C1_{r}_f1"]).max() <= 1e-4 * fmax
        assert np.abs(sc["f2"] - fc1[f"C1_{r}_f2"]).max() <= 1e-4 * fmax
    dda.release()


# ---- periodic targets (IPBC = 1) against tests/golden/reference_fixtures_pbc.npz;
# the inputs are regenerated by tests/golden/edge_cases.py
FIX_PBC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_pbc.npz")


def _edge_cases():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import edge_cases
    return edge_cases


@pytest.fixture(scope="module")
def fpbc():
    return dict(np.load(FIX_PBC))


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
@pytest.mark.parametrize("case", ["y", "z", "yz", "yf"])
def test_periodic_matvec_vs_reference(fpbc, case, layout):
    """Periodicity in y (JPBC 1), z (JPBC 2), y and z (JPBC 3), and in y with
    IDIPINT = 1: the replica-sum Green build and the full-tensor MATVEC."""
    cs = {c["name"]: c for c in _edge_cases().pbc_cases()}[case]
    dda = D.DDA(layout)
    dda.prepare_green(*cs["dims"], cs["iocc"], cs["ak"], ipbc=1, idipint=cs["idipint"], gamma=cs["gamma"],
                      pyd=cs["pyd"], pzd=cs["pzd"])
    for cw in "NC":
        y = dda.apply(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fpbc[f"M_{case}_y{cw}"]) < 2e-5
        assert np.all(y.reshape(3, -1)[:, cs["iocc"] == 0] == 0)
    dda.release()


@pytest.mark.gpu
def test_periodic_solve_evalq_scat_vs_reference(fpbc):
    """A slab periodic in y and z: PBCGS2 return code, ITNO, NCOMPTE and
    solution, EVALQ, and SCAT with JPBC = 3 (no finite-target integration:
    zero sums and NAVG = 0; amplitudes in the selected directions, within
    2e-5 of the largest)."""
    prob, gamma, pyd, pzd, aks, em1, em2 = _edge_cases().pbc_solve_problem()
    k = prob.incid[0].k.astype(np.float32)
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, k, ipbc=1, gamma=gamma, pyd=pyd, pzd=pzd)
    out = dda.solve("pbcgs2", prob.rhs(0), prob.adia(0), prob.aoff(), maxit=300, tol=TOL, check=False)
    it_ref, tole_ref, nc_ref = fpbc["P_meta"]
    assert out.rc == int(fpbc["P_rc"][0]) == 0 and out.tole <= TOL
    assert abs(out.itno - it_ref) <= 1 and abs(out.ncompte - nc_ref) <= 2, (out.itno, out.ncompte)
    assert _rel(out.x, fpbc["P_x"]) < 20 * TOL
    for g, r in zip(dda.evalq(k), fpbc["P_evalq"]):
        assert abs(g - r) <= 1e-5 * abs(r)
    sc = dda.scat(k, prob.incid[0].e, prob.x0, etasca=0.0, jpbc=3, aks=aks, em1=em1, em2=em2)
    assert sc["navg"] == 0 and sc["csca"] == 0.0 and sc["cbksca"] == 0.0 and sc["cscag2"] == 0.0
    fmax = np.abs(fpbc["P_f1"]).max()
    assert np.abs(sc["f1"] - fpbc["P_f1"]).max() <= 2e-5 * fmax
    assert np.abs(sc["f2"] - fpbc["P_f2"]).max() <= 2e-5 * fmax
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
def test_periodic_prepare_f32_vs_reference(fpbc, layout):
    """ddscat_cuda_prepare_f32 with IPBC = 1 and a caller-supplied full-grid
    spectrum (planar, six components), then the MATVEC in both CWHAT."""
    cs = _edge_cases().pbc_cpu_green_case()
    dda = D.DDA(layout)
    dda.prepare(*cs["dims"], cs["iocc"], cs["green"], ipbc=1)
    for cw in "NC":
        y = dda.apply(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fpbc[f"M_cpu_y{cw}"]) < 2e-5
    dda.release()


# ---- rectangular lattices (dx1..dx3 = 1.0, 0.9, 1.1) against
# tests/golden/reference_fixtures_dx.npz
FIX_DX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_dx.npz")


@pytest.fixture(scope="module")
def fdx():
    return dict(np.load(FIX_DX))


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
@pytest.mark.parametrize("case", ["iso", "flt", "pbc"])
def test_rectangular_lattice_matvec_vs_reference(fdx, case, layout):
    EC = _edge_cases()
    cs = {c["name"]: c for c in EC.dx_cases()}[case]
    dda = D.DDA(layout)
    dda.prepare_green(*cs["dims"], cs["iocc"], cs["ak"], dx=EC.DX, ipbc=cs["ipbc"], idipint=cs["idipint"],
                      gamma=cs["gamma"], pyd=cs["pyd"], pzd=0.0)
    for cw in "NC":
        y = dda.apply(cs["x"], cs["adia"], cs["aoff"], cw)
        assert _rel(y, fdx[f"M_{case}_y{cw}"]) < 2e-5
    dda.release()


@pytest.mark.gpu
def test_rectangular_lattice_solve_evalq_scat_vs_reference(fdx):
    """QMRCCG on an ellipsoid of the rectangular lattice (the padded register-FFT
    grid), EVALQ, and SCAT with the site positions ((i+1)+x0)*DX."""
    EC = _edge_cases()
    prob, aks, em1, em2 = EC.dx_solve_problem()
    k = prob.incid[0].k.astype(np.float32)
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, k, dx=EC.DX)
    out = dda.solve("qmrccg", prob.rhs(0), prob.adia(0), prob.aoff(), maxit=300, tol=TOL)
    it_ref, tole_ref, nc_ref = fdx["Q_meta"]
    assert out.rc == int(fdx["Q_rc"][0]) == 0 and out.tole <= TOL
    assert abs(out.itno - it_ref) <= max(1, 0.2 * it_ref) and abs(out.ncompte - nc_ref) <= max(2, 0.2 * nc_ref)
    assert _rel(out.x, fdx["Q_x"]) < 20 * TOL
    for g, r in zip(dda.evalq(k), fdx["Q_evalq"]):
        assert abs(g - r) <= 1e-5 * abs(r)
    sc = dda.scat(k, prob.incid[0].e, prob.x0, dx=EC.DX, etasca=3.0, aks=aks, em1=em1, em2=em2)
    cb, cs, g0, g1, g2, cg2, navg = fdx["Q_scat"]
    assert sc["navg"] == int(navg)
    assert abs(sc["csca"] - cs) <= 1e-5 * cs and abs(sc["cscag2"] - cg2) <= 1e-5 * cs
    for a, r in zip(sc["cscag"], (g0, g1, g2)):
        assert abs(a - r) <= 1e-5 * cs
    assert abs(sc["cbksca"] - cb) <= 1e-5 * cs
    fmax = np.abs(fdx["Q_f1"]).max()
    assert np.abs(sc["f1"] - fdx["Q_f1"]).max() <= 2e-5 * fmax
    assert np.abs(sc["f2"] - fdx["Q_f2"]).max() <= 2e-5 * fmax
    dda.release()


# ---- limit cases of all eight solvers against tests/golden/reference_fixtures_limits.npz
FIX_LIM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_fixtures_limits.npz")


@pytest.fixture(scope="module")
def flim():
    return dict(np.load(FIX_LIM))


@pytest.mark.gpu
@pytest.mark.parametrize("name", D.SOLVERS)
def test_solver_limits_vs_reference(flim, name):
    """MAXIT reached (maxit 3, tol 1e-12), a zero right-hand side and a nonzero
    initial guess: the same return code, ITNO and NCOMPTE as the reference, TOLE
    within 2 % + 1e-7 (FP32 stagnation near 1e-6 after three BiCGStab(4) steps
    varies by a few per cent; both 0 or inf on the early exits), and the same
    iterate."""
    prob, b, adia, aoff, x0 = _edge_cases().limits_problem()
    dda = D.DDA()
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k.astype(np.float32))
    for tag, bb, xx, maxit, tol in (("maxit", b, None, 3, 1e-12), ("zero", np.zeros_like(b), None, 10, 1e-5),
                                    ("x0", b, x0, 300, 1e-5)):
        out = dda.solve(name, bb, adia, aoff, x0=xx, maxit=maxit, tol=tol, check=False)
        it_ref, tole_ref, nc_ref = flim[f"L_{name}_{tag}_meta"]
        assert out.rc == int(flim[f"L_{name}_{tag}_rc"][0]), (tag, out.rc)
        assert out.itno == int(it_ref) and out.ncompte == int(nc_ref), (tag, out.itno, out.ncompte)
        if np.isfinite(tole_ref) and tole_ref > 0:
            assert abs(out.tole - tole_ref) <= 0.02 * tole_ref + 1e-7, (tag, out.tole, tole_ref)
        else:
            assert out.tole == tole_ref, (tag, out.tole, tole_ref)
        xr = flim[f"L_{name}_{tag}_x"]
        if np.linalg.norm(xr) > 0:
            assert _rel(out.x, xr) < 2 * TOL, tag
        else:
            assert np.all(out.x == 0), tag
    dda.release()
