"""Full-size checks of the 256^3 configuration (sphere, m = 1.6+0.02i, x = 60,
NAT = 16.8 M) in both layouts, through size-independent properties:

* the FFT3D and SLICES libraries give the same MATVEC (relative L2 <= 1e-6:
  same arithmetic, different middle-stage batching);
* the operator is complex symmetric: x2^T (A x1) = x1^T (A x2) to FP32
  accuracy (relative 1e-5);
* PBCGS2 through the reference ABI converges in both layouts, the FP64 true
  residual of each solution is <= 1.2*TOL and the two solutions agree to
  20*TOL."""
import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets

TOL = 1e-5
N = 256


@pytest.fixture(scope="module")
def prob():
    return targets.make_problem(N, m=1.6 + 0.02j, x=60.0)


def _rel(a, b):
    return float(np.linalg.norm((a - b).astype(np.complex128)) / np.linalg.norm(b.astype(np.complex128)))


@pytest.mark.gpu
def test_256_layouts_agree_and_operator_symmetric(prob):
    rng = np.random.default_rng(21)
    n3 = 3 * prob.nat
    occ3 = np.tile(prob.iocc != 0, 3)
    xs = []
    for _ in range(2):
        v = (rng.normal(size=n3) + 1j * rng.normal(size=n3)).astype(np.complex64)
        v[~occ3] = 0
        xs.append(v)
    adia = prob.adia(0)
    aoff = np.zeros(n3, dtype=np.complex64)
    ys = {}
    for layout in ("fft3d", "slices"):
        dda = D.DDA(layout)
        dda.prepare_green(N, N, N, prob.iocc, prob.incid[0].k)
        ys[layout] = [dda.apply(v, adia, aoff) for v in xs]
        dda.release()
    for a, b in zip(ys["slices"], ys["fft3d"]):
        assert _rel(a, b) <= 1e-6
    y1, y2 = ys["fft3d"]
    s12 = np.dot(xs[1].astype(np.complex128), y1.astype(np.complex128))
    s21 = np.dot(xs[0].astype(np.complex128), y2.astype(np.complex128))
    scale = np.linalg.norm(xs[1].astype(np.complex128)) * np.linalg.norm(y1.astype(np.complex128))
    assert abs(s12 - s21) <= 1e-5 * scale


@pytest.mark.gpu
def test_256_pbcgs2_both_layouts(prob):
    b = prob.rhs(0)
    adia = prob.adia(0)
    aoff = prob.aoff()
    sols = {}
    for layout in ("fft3d", "slices"):
        dda = D.DDA(layout)
        dda.prepare_green(N, N, N, prob.iocc, prob.incid[0].k)
        out = dda.solve("pbcgs2", b, adia, aoff, maxit=2000, tol=TOL)
        assert out.tole <= TOL, (layout, out.itno, out.tole)
        r64 = dda.residual_f64(b[None, :], out.x[None, :], adia[None, :])
        assert r64[0] <= 1.2 * TOL, (layout, r64)
        sols[layout] = out.x
        dda.release()
    assert _rel(sols["slices"], sols["fft3d"]) < 20 * TOL
