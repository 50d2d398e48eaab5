"""The allocation-free MATVEC entry point, ddscat_b200_apply_noalloc_f32.

It exists for callers that cannot allocate device memory where they need the
operator: real-time loops that forbid allocation once they run, and
applications that give all device memory to their own pool.  It must return
the same y as ddscat_cuda_apply_f32 on the same inputs (FP32 tolerance 2e-5
relative, as in test_gpu_matvec.py) on two calls in a row, leave the free
device memory unchanged, and reject targets whose padded FFT grid does not fit
its fixed scratch.  This file is named to be collected last."""
import ctypes as ct

import numpy as np
import pytest

import ddscat_b200 as D

RTOL = 2e-5


def _inputs(dims, seed):
    rng = np.random.default_rng(seed)
    nat = int(np.prod(dims))
    iocc = (rng.random(nat) < 0.8).astype(np.int16)
    iocc[0] = 1
    ak = tuple(rng.normal(size=3) * 0.4)
    c = lambda s=1.0: (s * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)  # noqa: E731
    return iocc, ak, c(), c(), c(), c(0.3)


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 16, 16), (12, 10, 9), (18, 18, 18)])
def test_apply_noalloc_matches_apply(dims):
    """16^3: x-first pipeline with M = 2n; 12x10x9: z-first pipeline; 18^3: x-first
    on padded FFT lengths (36 -> 48)."""
    torch = pytest.importorskip("torch")
    iocc, ak, x1, x2, adia, aoff = _inputs(dims, 7)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    lib = dda.lib
    dev = torch.device("cuda", torch.cuda.current_device())
    xd1, xd2 = torch.from_numpy(x1).to(dev), torch.from_numpy(x2).to(dev)
    ad, od = torch.from_numpy(adia).to(dev), torch.from_numpy(aoff).to(dev)
    yd1, yd2 = torch.empty_like(xd1), torch.empty_like(xd1)
    p = lambda t: ct.c_void_p(t.data_ptr())  # noqa: E731
    # first call on this device: one-time set-up (scratch address lookup)
    assert lib.ddscat_b200_apply_noalloc_f32(ord("N"), p(xd1), p(yd1), p(ad), p(od), None) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    # two calls in a row, different inputs and CWHAT
    assert lib.ddscat_b200_apply_noalloc_f32(ord("N"), p(xd1), p(yd1), p(ad), p(od), None) == 0
    assert lib.ddscat_b200_apply_noalloc_f32(ord("C"), p(xd2), p(yd2), p(ad), p(od), None) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    for yd, xh, cw in ((yd1, x1, "N"), (yd2, x2, "C")):
        ref = dda.apply(xh, adia, aoff, cw)
        got = yd.cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= RTOL
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(16, 16, 16), (18, 18, 18)])
def test_apply_noalloc_in_cuda_graph(dims):
    """The call captured into a CUDA graph on a caller's stream: every replay
    reads the current contents of x and writes y, equal to ddscat_cuda_apply_f32
    on the same inputs (the kernels' parameters, tensor maps included, are fixed
    at capture; the scratch is the same fixed array)."""
    torch = pytest.importorskip("torch")
    iocc, ak, x1, x2, adia, aoff = _inputs(dims, 11)
    dda = D.DDA()
    dda.prepare_green(*dims, iocc, ak)
    lib = dda.lib
    dev = torch.device("cuda", torch.cuda.current_device())
    xd = torch.from_numpy(x1).to(dev)
    ad, od = torch.from_numpy(adia).to(dev), torch.from_numpy(aoff).to(dev)
    yd = torch.empty_like(xd)
    p = lambda t: ct.c_void_p(t.data_ptr())  # noqa: E731
    s = torch.cuda.Stream()
    sp = ct.c_void_p(s.cuda_stream)
    s.wait_stream(torch.cuda.current_stream())
    # uncaptured call first (one-time set-up), then the capture
    assert lib.ddscat_b200_apply_noalloc_f32(ord("N"), p(xd), p(yd), p(ad), p(od), sp) == 0
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(g, stream=s, capture_error_mode="thread_local"):
        rcs.append(lib.ddscat_b200_apply_noalloc_f32(ord("N"), p(xd), p(yd), p(ad), p(od), sp))
    assert rcs == [0]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    got = []
    for xh in (x2, x1):
        xd.copy_(torch.from_numpy(xh))
        yd.zero_()
        g.replay()
        torch.cuda.synchronize()
        got.append(yd.cpu().numpy())
    assert torch.cuda.mem_get_info()[0] == free0
    del g
    for xh, y in zip((x2, x1), got):
        ref = dda.apply(xh, adia, aoff, "N")
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= RTOL
    dda.release()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(72, 72, 72), (72, 72, 64)])
def test_apply_noalloc_rejects_large_target(dims):
    """72^3 has NAT = 373,248 > 349,525; 72x72x64 (NAT = 331,776) is under that
    bound but its x and y axes are padded from 144 to 192, so its scratch
    (9.7 M complex floats) exceeds the fixed 6.29 M as well."""
    torch = pytest.importorskip("torch")
    nat = int(np.prod(dims))
    dda = D.DDA()
    dda.prepare_green(*dims, np.ones(nat, dtype=np.int16), (0.3, 0.0, 0.0))
    t = torch.zeros(3 * nat, dtype=torch.complex64, device="cuda")
    p = ct.c_void_p(t.data_ptr())
    rc = dda.lib.ddscat_b200_apply_noalloc_f32(ord("N"), p, p, p, None, None)
    assert rc == 601
    assert b"at most" in dda.lib.ddscat_cuda_last_error()
    dda.release()
