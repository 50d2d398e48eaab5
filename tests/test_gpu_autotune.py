"""FFT launch-shape autotuner (ddscat_b200_autotune_f32): on grids that run the
z-first pipeline (non-power-of-two and mixed axes) it picks launch shapes, on
grids of the x-first pipeline (24^3: 48-point axes; 32x24x16) it picks between
the two z passes; the choice is never slower than the default (the default is
a candidate) and the MATVEC still matches the FP64 oracle (relative L2 <= 2e-5)."""
import numpy as np
import pytest

import ddscat_b200 as D
from oracle import ddscat_oracle as O


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(24, 24, 24), (15, 27, 20), (32, 24, 16)])
def test_autotune_keeps_parity(dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(8)
    nat = nx * ny * nz
    iocc = (rng.random(nat) < 0.7).astype(np.int16)
    ak = (0.3, -0.2, 0.25)
    x = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    adia = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    aoff = np.zeros(3 * nat, dtype=np.complex64)
    dda = D.DDA()
    dda.prepare_green(nx, ny, nz, iocc, ak)
    d, b = dda.autotune(iters=3)
    assert 0 < b <= d
    y = dda.apply(x, adia, aoff)
    gp = O.GreenParams(nx, ny, nz, ak=tuple(float(np.float32(a)) for a in ak))
    yr = O.Operator.from_params(gp, iocc).apply_full(x, adia, aoff)
    assert np.linalg.norm(y - yr) / np.linalg.norm(yr) <= 2e-5
    dda.release()
