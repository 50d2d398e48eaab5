"""DDSCAT's own path into the library, on the GPU: the reference's C loader
(compiled unmodified) and a C stand-in for the Fortran bridge
(oracle/_ref/ddscat_bridge_driver, see oracle/bridge_driver.c) run
prepare_green -> solver -> EVALQ (resident solution) -> SCAT -> release
against each of this project's libraries, selected with DDSCAT_CUDA_DLL as
DDSCAT selects it.  The results are checked against the FP64 oracle: the
solution's FP64 true residual <= 1.2 tol, EVALQ 1e-6 and SCAT's Csca, g and
f1/f2 1e-5 relative, evaluated by the oracle on the returned solution."""
import os
import subprocess

import numpy as np
import pytest

from ddscat_b200 import targets
from oracle import ddscat_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ddscat_bridge_driver")
LIBS = {"fft3d": "libddscat_matvec_cuda.so", "slices": "libddscat_matvec_cuda_slice.so"}
SOLVER_IDS = {"gpbicg": 0, "qmrccg": 1, "pbcgst": 2, "pbcgs2": 3, "petrkp": 4}
TOL = 1e-5


def _write_input(path, prob, r, solver, aks, em1, em2, etasca=0.5, maxit=500):
    k = prob.incid[r].k.astype(np.float32)
    ndir = aks.shape[0]
    hdr_i = np.array([prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, SOLVER_IDS[solver], maxit, ndir],
                     dtype=np.int32)
    hdr_f = np.array([0.0, 0.0, 0.0, *k, 1.0, 1.0, 1.0, TOL, etasca, 1.0, *prob.x0], dtype=np.float32)
    with open(path, "wb") as f:
        for a in (hdr_i, hdr_f, prob.iocc.astype(np.int16), prob.rhs(r), prob.adia(r), prob.aoff(),
                  prob.incid[r].e.astype(np.complex64), aks.astype(np.float32), em1.astype(np.float32),
                  em2.astype(np.float32)):
            f.write(np.ascontiguousarray(a).tobytes())


def _read_output(path, nat, ndir):
    raw = open(path, "rb").read()
    ints = np.frombuffer(raw, np.int32, 8, 0)
    tole = float(np.frombuffer(raw, np.float32, 1, 32)[0])
    q = np.frombuffer(raw, np.float64, 9, 36)
    off = 36 + 72
    x = np.frombuffer(raw, np.complex64, 3 * nat, off)
    f1 = np.frombuffer(raw, np.complex64, ndir, off + 24 * nat)
    f2 = np.frombuffer(raw, np.complex64, ndir, off + 24 * nat + 8 * ndir)
    return ints, tole, q, x, f1, f2


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
@pytest.mark.parametrize("solver", ["pbcgs2", "qmrccg"])
def test_bridge_sequence_through_reference_loader(tmp_path, layout, solver):
    if not os.path.exists(DRIVER):
        pytest.skip("bridge driver not built (oracle/Makefile)")
    n = 16
    prob = targets.make_problem(n, m=1.5 + 0.01j, x=3.0)
    r = 1
    k = prob.incid[r].k
    aks, em1, em2 = targets.scattering_planes(k, prob.incid[r].e, step_deg=10.0)
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    _write_input(fin, prob, r, solver, aks, em1, em2)
    env = dict(os.environ, DDSCAT_CUDA_DLL=os.path.join(ROOT, "ddscat-cuda_b200", "lib", LIBS[layout]))
    run = subprocess.run([DRIVER, "run", str(fin), str(fout)], env=env, capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stderr
    assert "DDSCAT CUDA library loaded" in run.stdout
    ints, tole, q, x, f1, f2 = _read_output(fout, prob.nat, aks.shape[0])
    assert list(ints[:5]) == [0, 0, 0, 0, 0], (ints, run.stderr)
    itno, ncompte, navg = ints[5:]
    assert itno > 0 and ncompte >= itno and tole <= TOL
    # the oracle on the returned solution
    op = O.Operator.from_params(O.GreenParams(n, n, n, ak=tuple(float(np.float32(a)) for a in k)), prob.iocc)
    occ = op.occ
    bc = O.gather_compact(prob.rhs(r), occ, prob.nat).astype(np.complex128)
    ac = O.gather_compact(prob.adia(r), occ, prob.nat).astype(np.complex128)
    zero = np.zeros_like(ac)
    xc = O.gather_compact(x, occ, prob.nat).astype(np.complex128)
    true = np.linalg.norm(bc - op.apply_compact(xc, ac, zero)) / np.linalg.norm(bc)
    assert true <= 1.2 * TOL
    assert np.all(x.reshape(3, -1)[:, prob.iocc == 0] == 0)
    cabs, cext, cpha = O.evalq(bc, xc, ac, zero, k, 1.0)
    for got, want in zip(q[:3], (cabs, cext, cpha)):
        assert abs(got - want) <= 1e-6 * abs(want)
    sc = O.scat(xc, occ, n, n, 0, k, aks, (1.0, 1.0, 1.0), em1, em2, 1.0, 0.5, prob.incid[r].e, prob.x0)
    assert navg == sc["navg"]
    assert q[4] == pytest.approx(sc["csca"], rel=1e-5)
    assert q[5] / q[4] == pytest.approx(sc["cscag"][0] / sc["csca"], abs=1e-5)
    fmax = max(np.abs(sc["f1"]).max(), np.abs(sc["f2"]).max())
    assert np.abs(f1 - sc["f1"]).max() <= 1e-5 * fmax and np.abs(f2 - sc["f2"]).max() <= 1e-5 * fmax
