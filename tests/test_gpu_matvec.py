"""GPU parity of the MATVEC and the Green build against the FP64 oracle,
through the C ABI (ddscat_cuda_prepare_green_f32 / prepare_f32 / apply_f32).

Tolerance: complex-FP32 bulk arithmetic, so the relative L2 error of y must be
<= 2e-5 and the max-norm error <= 1e-4 of max|y| (the FFT error grows like
eps_f32 * log2(M))."""
import numpy as np
import pytest

import ddscat_b200 as D
from oracle import ddscat_oracle as O

RTOL_L2 = 2e-5
RTOL_MAX = 1e-4


def _case(dims, idipint, seed=11, occ_p=0.7):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    nat = nx * ny * nz
    iocc = (rng.random(nat) < occ_p).astype(np.int16)
    iocc[0] = 1
    ak = tuple(rng.normal(size=3) * 0.4)
    x = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    adia = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    aoff = (0.3 * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)
    gp = O.GreenParams(nx, ny, nz, idipint=idipint, ak=tuple(float(np.float32(a)) for a in ak))
    return iocc, ak, x, adia, aoff, gp


def _err(y, yr):
    l2 = np.linalg.norm(y - yr) / np.linalg.norm(yr)
    mx = np.abs(y - yr).max() / np.abs(yr).max()
    return l2, mx


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["fft3d", "slices"])
@pytest.mark.parametrize("dims,idipint", [((4, 4, 4), 0), ((5, 3, 4), 0), ((6, 5, 7), 1), ((7, 11, 13), 0),
                                          ((8, 8, 8), 0), ((12, 10, 9), 1), ((16, 16, 16), 0), ((24, 18, 30), 0),
                                          ((32, 32, 32), 0), ((16, 8, 32), 1), ((64, 32, 16), 0), ((8, 64, 16), 0),
                                          ((128, 16, 8), 1), ((64, 64, 64), 0),
                                          # 3 * 2^k padded lengths (x-first pipeline with 12/24-point DFTs)
                                          ((24, 24, 24), 0), ((48, 24, 96), 1), ((96, 32, 24), 0), ((48, 48, 48), 0),
                                          # even n whose 2n is no register-FFT length: padded FFT lengths
                                          # (40, 52, 28 -> 48, 64, 32; 100, 20, 60 -> 128, 32, 64)
                                          ((20, 26, 14), 1), ((50, 10, 30), 0),
                                          # (M_x, M_y) = (256, 256), (128, 256), (256, 128), full and padded rows
                                          ((128, 128, 8), 0), ((100, 120, 6), 1), ((64, 128, 10), 0),
                                          ((128, 60, 8), 0),
                                          # 512-point passes: z (kx_zg, E = 32), x and y (two TMA boxes per tile)
                                          ((8, 8, 200), 0), ((200, 6, 8), 1), ((6, 200, 8), 0)])
def test_apply_matches_oracle(layout, dims, idipint):
    iocc, ak, x, adia, aoff, gp = _case(dims, idipint)
    dda = D.DDA(layout)
    dda.prepare_green(*dims, iocc, ak, idipint=idipint)
    op = O.Operator.from_params(gp, iocc)
    for cwhat in "NC":
        y = dda.apply(x, adia, aoff, cwhat)
        yr = op.apply_full(x, adia, aoff, cwhat)
        l2, mx = _err(y, yr)
        assert l2 <= RTOL_L2 and mx <= RTOL_MAX, (cwhat, l2, mx)
        # unoccupied sites are exactly zero (cu:117)
        assert np.all(y.reshape(3, -1)[:, iocc == 0] == 0)
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(10, 9, 8), (16, 8, 8)])
def test_prepare_with_cpu_green_matches_gpu_green(dims):
    iocc, ak, x, adia, aoff, gp = _case(dims, 0, seed=5)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    y1 = dda.apply(x, adia, aoff)
    oct6 = O.green_octant(gp).astype(np.complex64)
    dda.prepare(*dims, iocc, oct6)
    y2 = dda.apply(x, adia, aoff)
    yr = O.Operator.from_octant(*dims, oct6.astype(np.complex128), iocc).apply_full(x, adia, aoff)
    assert _err(y2, yr)[0] <= RTOL_L2
    assert _err(y1, y2)[0] <= RTOL_L2
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(4, 3, 3), (8, 8, 8)])
def test_pbc_green_matches_oracle(dims):
    """IPBC=1 (periodic in y): full-tensor Green build and MATVEC branch
    (a generic-length grid and a power-of-two grid)."""
    rng = np.random.default_rng(2)
    nat = int(np.prod(dims))
    iocc = np.ones(nat, dtype=np.int16)
    ak = (0.6, 0.25, 0.0)
    x = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    adia = np.full(3 * nat, 2.0 + 0.5j, dtype=np.complex64)
    aoff = np.zeros(3 * nat, dtype=np.complex64)
    gamma, pyd = 5e-2, 3.0
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak, ipbc=1, gamma=gamma, pyd=pyd, pzd=0.0)
    y = dda.apply(x, adia, aoff)
    gp = O.GreenParams(*dims, ipbc=1, gamma=gamma, pyd=pyd, pzd=0.0,
                       ak=tuple(float(np.float32(a)) for a in ak))
    op = O.Operator.from_params(gp, iocc)
    yr = op.apply_full(x, adia, aoff)
    assert _err(y, yr)[0] <= 1e-4
    dda.release()


@pytest.mark.gpu
def test_apply_is_linear_and_symmetric():
    """Size-independent properties at a larger grid: A(a x + b z) = a Ax + b Az
    and z^T A x = x^T A z (complex symmetry)."""
    dims = (40, 36, 32)
    iocc, ak, x, adia, aoff, gp = _case(dims, 0, seed=3, occ_p=1.0)
    rng = np.random.default_rng(4)
    z = (rng.normal(size=x.size) + 1j * rng.normal(size=x.size)).astype(np.complex64)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    ax, az = dda.apply(x, adia, aoff), dda.apply(z, adia, aoff)
    a, b = 0.3 - 0.7j, 1.1 + 0.2j
    lin = dda.apply((a * x + b * z).astype(np.complex64), adia, aoff)
    assert np.linalg.norm(lin - (a * ax + b * az)) / np.linalg.norm(lin) < 5e-6
    s1 = np.dot(z.astype(np.complex128), ax.astype(np.complex128))
    s2 = np.dot(x.astype(np.complex128), az.astype(np.complex128))
    assert abs(s1 - s2) / abs(s1) < 1e-5
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(20, 26, 14), (40, 36, 32)])
def test_padded_fft_lengths_equal_2n(dims, monkeypatch):
    """With a library-built Green tensor, even grids whose 2n is no register-FFT
    length run on padded FFT lengths (next register length >= 2n); the operator
    equals the one on the 2n grid (DDSCAT_B200_NOPAD=1) to FP32 rounding."""
    iocc, ak, x, adia, aoff, gp = _case(dims, 0, seed=6)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    y_pad = dda.apply(x, adia, aoff)
    monkeypatch.setenv("DDSCAT_B200_NOPAD", "1")
    dda.prepare_green(*dims, iocc, ak)
    y_2n = dda.apply(x, adia, aoff)
    assert _err(y_pad, y_2n)[0] <= 1e-5
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(32, 32, 12), (64, 64, 20), (120, 128, 16)])
def test_fused_xy_passes_equal_five_pass(dims, monkeypatch):
    """With DDSCAT_B200_FUSEXY=1, FP32 grids with (M_x, M_y) in the fused set
    run the x and y passes of a z plane in one four-CTA cluster (distributed
    shared memory, B laid out ky-contiguous): the same transforms in the same
    order as the five-pass schedule, so both give the same y to rounding, for
    'N' and 'C' and with CXAOFF."""
    iocc, ak, x, adia, aoff, gp = _case(dims, 0, seed=9)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    y_5 = [dda.apply(x, adia, aoff, cw) for cw in "NC"]
    monkeypatch.setenv("DDSCAT_B200_FUSEXY", "1")
    y_f = [dda.apply(x, adia, aoff, cw) for cw in "NC"]
    for a, b in zip(y_f, y_5):
        assert _err(a, b)[0] <= 1e-6
    dda.release()


@pytest.mark.gpu
def test_slices_uneven_middle_batches_equal_fft3d():
    """SLICES with middle-stage batches of unequal size: at 128 x 128 x 64 the
    32 MiB floor gives batches of 86, 86 and 84 kx planes (the last one
    shorter); the MATVEC equals the FFT3D layout's, whose middle stage holds
    every plane at once, to FP32 rounding, in both CWHAT."""
    dims = (128, 128, 64)
    iocc, ak, x, adia, aoff, gp = _case(dims, 0, seed=21)
    outs = {}
    for layout in ("fft3d", "slices"):
        dda = D.DDA(layout)
        dda.prepare_green(*dims, iocc, ak)
        outs[layout] = [dda.apply(x, adia, aoff, cw) for cw in "NC"]
        dda.release()
    for a, b in zip(outs["slices"], outs["fft3d"]):
        assert np.linalg.norm(a - b) / np.linalg.norm(b) <= 1e-6
