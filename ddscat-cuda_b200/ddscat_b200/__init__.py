"""Thin ctypes binding of the B200 DDA library (used by tests and bench).

It calls the C ABI declared in ``include/ddscat_matvec_cuda.h`` and
``include/ddscat_b200.h`` with host NumPy arrays, the same way the DDSCAT
Fortran bridge does (``ddscat_cuda_unified/fortran/cuda_matvec_bridge.f90``):
full-grid component-major complex64 vectors of length 3*NAT.  There is no CPU
fallback: if the CUDA library is not built, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as ct
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_DIR = os.path.join(ROOT_DIR, "lib")
LIB_NAMES = {"fft3d": "libddscat_matvec_cuda.so", "slices": "libddscat_matvec_cuda_slice.so"}

SOLVERS = ("gpbicg", "qmrccg", "pbcgst", "pbcgs2", "petrkp", "bicgstab4", "gpbicgstab2", "gpbicgstab4")

# every symbol the C headers declare (checked by the CPU test suite)
EXPORTS = (
    ["ddscat_cuda_prepare_green_f32", "ddscat_cuda_prepare_f32", "ddscat_cuda_apply_f32"]
    + [f"ddscat_cuda_solve_{s}_f32" for s in SOLVERS]
    + ["ddscat_cuda_evalq_f32", "ddscat_cuda_scat_f32", "ddscat_cuda_release", "ddscat_cuda_last_error"]
    + ["ddscat_b200_set_verbose", "ddscat_b200_layout", "ddscat_b200_matvec_timing", "ddscat_b200_solve_batch_f32",
       "ddscat_b200_last_solve_stats", "ddscat_b200_residual_f64", "ddscat_b200_launch_count",
       "ddscat_b200_apply_noalloc_f32", "ddscat_b200_mueller_f32", "ddscat_b200_make_inputs_f32",
       "ddscat_b200_solve_batch_f64", "ddscat_b200_adjoint_f32", "ddscat_b200_multi_solve_f32",
       "ddscat_b200_autotune_f32", "ddscat_b200_mueller_f64", "ddscat_b200_scat_amplitudes_f64",
       "ddscat_b200_scat_csca_f64", "ddscat_b200_make_inputs_pol_f32", "ddscat_b200_adjoint_fwd_f32",
       "ddscat_b200_ffweights_f32", "ddscat_b200_scat_torque_f32"]
)


class DDSCATError(RuntimeError):
    def __init__(self, where, code, msg):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code
        self.msg = msg


def lib_path(layout="fft3d"):
    return os.path.join(LIB_DIR, LIB_NAMES[layout])


_P = ct.c_void_p
_I = ct.c_int
_F = ct.c_float
_D = ct.POINTER(ct.c_double)
_D2 = ct.c_double


def _declare(lib):
    f = lib.ddscat_cuda_prepare_green_f32
    f.argtypes = [_I] * 7 + [_F] * 9 + [_P]
    f.restype = _I
    f = lib.ddscat_cuda_prepare_f32
    f.argtypes = [_I] * 6 + [_P, _P]
    f.restype = _I
    f = lib.ddscat_cuda_apply_f32
    f.argtypes = [_I, _P, _P, _P, _P]
    f.restype = _I
    for s in SOLVERS:
        f = getattr(lib, f"ddscat_cuda_solve_{s}_f32")
        f.argtypes = [_P, _P, _P, _P, _I, _I, _F, ct.POINTER(_I), ct.POINTER(_F), ct.POINTER(_I)]
        f.restype = _I
    f = lib.ddscat_cuda_evalq_f32
    f.argtypes = [_I, _P, _P, _P, _P, _F, _F, _F, _F, _D, _D, _D]
    f.restype = _I
    f = lib.ddscat_cuda_scat_f32
    f.argtypes = [_I, _I, _P, _P, _P, _P, _P, _F, _F, _P, _P, _D, _D, _D, _D, ct.POINTER(_I), _P, _P]
    f.restype = _I
    lib.ddscat_cuda_release.argtypes = []
    lib.ddscat_cuda_release.restype = _I
    lib.ddscat_cuda_last_error.argtypes = []
    lib.ddscat_cuda_last_error.restype = ct.c_char_p
    lib.ddscat_b200_set_verbose.argtypes = [_I]
    lib.ddscat_b200_set_verbose.restype = _I
    lib.ddscat_b200_layout.argtypes = []
    lib.ddscat_b200_layout.restype = _I
    lib.ddscat_b200_matvec_timing.argtypes = [_I, _I, _I, ct.POINTER(_F)]
    lib.ddscat_b200_matvec_timing.restype = _I
    lib.ddscat_b200_solve_batch_f32.argtypes = [_I, _I, _P, _P, _P, _P, _I, _F, _P, _P, _P, _P]
    lib.ddscat_b200_solve_batch_f32.restype = _I
    lib.ddscat_b200_last_solve_stats.argtypes = [_D, ct.POINTER(ct.c_longlong), ct.POINTER(_I)]
    lib.ddscat_b200_last_solve_stats.restype = _I
    lib.ddscat_b200_residual_f64.argtypes = [_I, _P, _P, _P, _P, _D]
    lib.ddscat_b200_residual_f64.restype = _I
    lib.ddscat_b200_apply_noalloc_f32.argtypes = [_I, _P, _P, _P, _P, _P]
    lib.ddscat_b200_apply_noalloc_f32.restype = _I
    lib.ddscat_b200_mueller_f32.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D]
    lib.ddscat_b200_mueller_f32.restype = _I
    lib.ddscat_b200_make_inputs_f32.argtypes = [_I, _P, _P, _P, _I, _P, _P, _P, _P]
    lib.ddscat_b200_make_inputs_f32.restype = _I
    lib.ddscat_b200_make_inputs_pol_f32.argtypes = [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P]
    lib.ddscat_b200_make_inputs_pol_f32.restype = _I
    lib.ddscat_b200_adjoint_fwd_f32.argtypes = [_I, _P, _P, _P, _P, _I, _F, _P, _P, _P, _P]
    lib.ddscat_b200_adjoint_fwd_f32.restype = _I
    lib.ddscat_b200_ffweights_f32.argtypes = [_I, _P, _P, _P, _D2, _P]
    lib.ddscat_b200_ffweights_f32.restype = _I
    lib.ddscat_b200_solve_batch_f64.argtypes = [_I, _I, _P, _P, _P, _P, _I, _D2, _P, _P, _P, _P]
    lib.ddscat_b200_solve_batch_f64.restype = _I
    lib.ddscat_b200_adjoint_f32.argtypes = [_I, _P, _P, _P, _P, _I, _F, _P, _P, _P, _P]
    lib.ddscat_b200_adjoint_f32.restype = _I
    lib.ddscat_b200_multi_solve_f32.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _I, _I, _F, _I, _P, _P, _P, _P]
    lib.ddscat_b200_multi_solve_f32.restype = _I
    lib.ddscat_b200_autotune_f32.argtypes = [_I, _P, _P]
    lib.ddscat_b200_autotune_f32.restype = _I
    lib.ddscat_b200_mueller_f64.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _D]
    lib.ddscat_b200_mueller_f64.restype = _I
    lib.ddscat_b200_scat_amplitudes_f64.argtypes = [_I, _P, _I, _P, _P, _P, _P, _P, _P, _D2, _P, _P]
    lib.ddscat_b200_scat_amplitudes_f64.restype = _I
    lib.ddscat_b200_scat_csca_f64.argtypes = [_I, _P, _P, _P, _F, _P, _P, _F, _P, _P, _P, _P, _P]
    lib.ddscat_b200_scat_csca_f64.restype = _I
    lib.ddscat_b200_scat_torque_f32.argtypes = [_P, _P, _F, _F, _P, _P, _P, _P, ct.POINTER(_I)]
    lib.ddscat_b200_scat_torque_f32.restype = _I
    lib.ddscat_b200_launch_count.argtypes = []
    lib.ddscat_b200_launch_count.restype = ct.c_ulonglong


_LIBS = {}


def load(layout="fft3d"):
    """Load (once) the built library for ``layout`` ('fft3d' or 'slices')."""
    if layout in _LIBS:
        return _LIBS[layout]
    path = lib_path(layout)
    if not os.path.exists(path):
        raise OSError(f"B200 DDA library not built: {path} is missing (run `make -C ddscat-cuda_b200`)")
    lib = ct.CDLL(path, mode=ct.RTLD_LOCAL)
    _declare(lib)
    _LIBS[layout] = lib
    return lib


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p) if a is not None else None


def _c64(a, n=None):
    a = np.ascontiguousarray(np.asarray(a), dtype=np.complex64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} elements, got {a.size}")
    return a


BATCH_SOLVERS = {"qmrccg": 1, "pbcgs2": 2}
REPLACE_RESIDUAL = 0x100  # DDSCAT_B200_REPLACE_RESIDUAL
QMR_SYMMETRIC = 0x200  # DDSCAT_B200_QMR_SYMMETRIC
INPUTS_F64 = 0x400  # DDSCAT_B200_INPUTS_F64
AUTOTUNE = 0x800  # DDSCAT_B200_AUTOTUNE
GRAPH = 0x1000  # DDSCAT_B200_GRAPH
CMDPOL = {"LATTDR": 0, "GKDLDR": 1, "FLTRCD": 2}  # DDSCAT_B200_LATTDR, _GKDLDR, _FLTRCD


def _vptr(a):
    """Pointer of a host NumPy array or of a CUDA tensor (``data_ptr()``)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ct.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ct.c_void_p)


@dataclass
class BatchOut:
    rc: int
    itno: np.ndarray
    tole: np.ndarray
    ncompte: np.ndarray
    status: np.ndarray


@dataclass
class SolveOut:
    rc: int
    x: np.ndarray
    itno: int
    tole: float
    ncompte: int


class DDA:
    """One prepared target on the current CUDA device (the library keeps a
    single global state, like the reference)."""

    takes_device_pointers = True  # the batched / adjoint entry points accept CUDA tensors

    def __init__(self, layout="fft3d"):
        self.lib = load(layout)
        self.layout = layout
        self.nat = self.nat0 = 0

    def _err(self):
        return self.lib.ddscat_cuda_last_error().decode(errors="replace")

    def _check(self, where, rc):
        if rc != 0:
            raise DDSCATError(where, rc, self._err())

    def prepare_green(self, nx, ny, nz, iocc, ak, dx=(1.0, 1.0, 1.0), ipbc=0, idipint=0, gamma=0.0, pyd=0.0, pzd=0.0,
                      nat=None, nat0=None):
        iocc = np.ascontiguousarray(np.asarray(iocc), dtype=np.int16)
        self.nat = nx * ny * nz if nat is None else nat
        self.nat0 = int(np.count_nonzero(iocc)) if nat0 is None else nat0
        rc = self.lib.ddscat_cuda_prepare_green_f32(nx, ny, nz, ipbc, self.nat, self.nat0, idipint, gamma, pyd, pzd,
                                                    float(ak[0]), float(ak[1]), float(ak[2]), float(dx[0]),
                                                    float(dx[1]), float(dx[2]), _ptr(iocc))
        self._check("prepare_green", rc)
        return rc

    def prepare(self, nx, ny, nz, iocc, green, ipbc=0):
        iocc = np.ascontiguousarray(np.asarray(iocc), dtype=np.int16)
        self.nat = nx * ny * nz
        self.nat0 = int(np.count_nonzero(iocc))
        g = _c64(green)
        rc = self.lib.ddscat_cuda_prepare_f32(nx, ny, nz, ipbc, self.nat, self.nat0, _ptr(g), _ptr(iocc))
        self._check("prepare", rc)
        return rc

    def apply(self, x, adia, aoff, cwhat="N"):
        n = 3 * self.nat
        x, adia, aoff = _c64(x, n), _c64(adia, n), _c64(aoff, n)
        y = np.empty(n, dtype=np.complex64)
        rc = self.lib.ddscat_cuda_apply_f32(ord(cwhat), _ptr(x), _ptr(y), _ptr(adia), _ptr(aoff))
        self._check("apply", rc)
        return y

    def solve(self, name, b, adia, aoff, x0=None, maxit=300, tol=1e-5, check=True):
        n = 3 * self.nat
        b, adia, aoff = _c64(b, n), _c64(adia, n), _c64(aoff, n)
        x = np.zeros(n, dtype=np.complex64) if x0 is None else _c64(x0, n).copy()
        it, tole, nc = _I(0), _F(0.0), _I(0)
        fn = getattr(self.lib, f"ddscat_cuda_solve_{name}_f32")
        rc = fn(_ptr(b), _ptr(x), _ptr(adia), _ptr(aoff), n, maxit, tol, ct.byref(it), ct.byref(tole), ct.byref(nc))
        if check:
            self._check(name, rc)
        return SolveOut(rc, x, it.value, float(tole.value), nc.value)

    def evalq(self, ak, e02=1.0, use_resident=1, e=None, p=None, adia=None, aoff=None):
        cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
        arrs = [None if a is None else _c64(a) for a in (e, p, adia, aoff)]
        rc = self.lib.ddscat_cuda_evalq_f32(use_resident, *[_ptr(a) for a in arrs], float(ak[0]), float(ak[1]),
                                            float(ak[2]), e02, ct.byref(cabs), ct.byref(cext), ct.byref(cpha))
        self._check("evalq", rc)
        return cabs.value, cext.value, cpha.value

    def scat(self, ak, e01, x0, dx=(1.0, 1.0, 1.0), etasca=0.5, e02=1.0, jpbc=0, aks=None, em1=None, em2=None):
        akf = np.ascontiguousarray(ak, dtype=np.float32)
        dxf = np.ascontiguousarray(dx, dtype=np.float32)
        x0f = np.ascontiguousarray(x0, dtype=np.float32)
        e01c = _c64(e01, 3)
        ndir = 0 if aks is None else int(np.asarray(aks).size // 3)
        aksf = None if aks is None else np.ascontiguousarray(aks, dtype=np.float32).reshape(-1)
        em1f = None if em1 is None else np.ascontiguousarray(em1, dtype=np.float32).reshape(-1)
        em2f = None if em2 is None else np.ascontiguousarray(em2, dtype=np.float32).reshape(-1)
        f1 = np.zeros(max(ndir, 1), dtype=np.complex64)
        f2 = np.zeros(max(ndir, 1), dtype=np.complex64)
        cb, cs, cg2 = ct.c_double(), ct.c_double(), ct.c_double()
        cg = (ct.c_double * 3)()
        navg = _I(0)
        rc = self.lib.ddscat_cuda_scat_f32(jpbc, ndir, _ptr(akf), _ptr(aksf), _ptr(dxf), _ptr(em1f), _ptr(em2f), e02,
                                           etasca, _ptr(e01c), _ptr(x0f), ct.byref(cb), ct.byref(cs),
                                           ct.cast(cg, _D), ct.byref(cg2), ct.byref(navg), _ptr(f1), _ptr(f2))
        self._check("scat", rc)
        return {"cbksca": cb.value, "csca": cs.value, "cscag": [cg[0], cg[1], cg[2]], "cscag2": cg2.value,
                "navg": navg.value, "f1": f1[:ndir], "f2": f2[:ndir]}

    def scat_torque(self, ak, e01, x0, dx=(1.0, 1.0, 1.0), etasca=0.5, e02=1.0):
        """Radiative torque cross sections of the resident solution (DDSCAT's
        DOTORQ): dict with ctrq_inc (incident-field torque), ctrq_flux (angular
        momentum carried off by the scattered light), ctrq = ctrq_inc - ctrq_flux
        (net), each a 3-vector in the frame of ak, and navg."""
        akf = np.ascontiguousarray(ak, dtype=np.float32)
        dxf = np.ascontiguousarray(dx, dtype=np.float32)
        x0f = np.ascontiguousarray(x0, dtype=np.float32)
        e01c = _c64(e01, 3)
        cinc, cflux = np.zeros(3), np.zeros(3)
        navg = _I(0)
        rc = self.lib.ddscat_b200_scat_torque_f32(_ptr(akf), _ptr(dxf), e02, etasca, _ptr(e01c), _ptr(x0f),
                                                  _ptr(cinc), _ptr(cflux), ct.byref(navg))
        self._check("scat_torque", rc)
        return {"ctrq_inc": cinc, "ctrq_flux": cflux, "ctrq": cinc - cflux, "navg": navg.value}

    def solve_batch(self, name, b, x, adia, aoff=None, maxit=300, tol=1e-5, check=True, replace=False,
                    symmetric=False, graph=False):
        """Batched solve; b, x (in/out), adia, aoff are (nrhs, 3*NAT) complex64
        host arrays, or CUDA tensors of the same shape (device-resident path).
        replace=True selects residual replacement instead of restarts at the
        reliable-residual checks; symmetric=True (QMRCCG) uses one MATVEC per
        iteration (left Lanczos vectors equal to the right ones); graph=True
        (QMRCCG with both, PBCGS2 with replace) runs the iterations
        device-driven as a CUDA graph."""
        nrhs = int(b.shape[0])
        for a in (b, x, adia) + (() if aoff is None else (aoff,)):
            if tuple(a.shape) != (nrhs, 3 * self.nat):
                raise ValueError(f"expected shape {(nrhs, 3 * self.nat)}, got {tuple(a.shape)}")
            if not hasattr(a, "data_ptr") and (a.dtype != np.complex64 or not a.flags.c_contiguous):
                raise ValueError("host arrays must be C-contiguous complex64")
        it = np.zeros(nrhs, dtype=np.int32)
        tole = np.zeros(nrhs, dtype=np.float32)
        nc = np.zeros(nrhs, dtype=np.int32)
        st = np.zeros(nrhs, dtype=np.int32)
        code = BATCH_SOLVERS[name] | (REPLACE_RESIDUAL if replace else 0) | (QMR_SYMMETRIC if symmetric else 0)
        code |= GRAPH if graph else 0
        rc = self.lib.ddscat_b200_solve_batch_f32(code, nrhs, _vptr(b), _vptr(x), _vptr(adia),
                                                  _vptr(aoff), maxit, tol, _ptr(it), _ptr(tole), _ptr(nc), _ptr(st))
        if check:
            self._check("solve_batch", rc)
        return BatchOut(rc, it, tole, nc, st)

    def solve_batch_f64(self, name, b, x, adia, aoff=None, maxit=1000, tol=1e-9, check=True, replace=False,
                        symmetric=False):
        """All-FP64 batched solve; b, adia, aoff complex64 or complex128
        (nrhs, 3*NAT), x complex128 (nrhs, 3*NAT) in/out; NumPy arrays or CUDA
        tensors."""
        nrhs = int(b.shape[0])
        in64 = str(b.dtype).endswith("complex128")
        for a in (adia,) + (() if aoff is None else (aoff,)):
            if str(a.dtype).endswith("complex128") != in64:
                raise ValueError("b, adia and aoff must share one precision")
        if not hasattr(x, "data_ptr") and (x.dtype != np.complex128 or not x.flags.c_contiguous):
            raise ValueError("x must be a C-contiguous complex128 array")
        it = np.zeros(nrhs, dtype=np.int32)
        tole = np.zeros(nrhs, dtype=np.float64)
        nc = np.zeros(nrhs, dtype=np.int32)
        st = np.zeros(nrhs, dtype=np.int32)
        code = BATCH_SOLVERS[name] | (REPLACE_RESIDUAL if replace else 0) | (QMR_SYMMETRIC if symmetric else 0)
        code |= INPUTS_F64 if in64 else 0
        rc = self.lib.ddscat_b200_solve_batch_f64(code, nrhs, _vptr(b), _vptr(x), _vptr(adia), _vptr(aoff), maxit,
                                                  float(tol), _ptr(it), _ptr(tole), _ptr(nc), _ptr(st))
        if check:
            self._check("solve_batch_f64", rc)
        return BatchOut(rc, it, tole, nc, st)

    def adjoint(self, p, src, adia, dadia, maxit=1000, tol=1e-5, want_lam=False):
        """Per-site derivatives of s^T P (see ddscat_b200_adjoint_f32); all
        arguments (nrhs, 3*NAT) complex64 NumPy arrays.  Returns (grad (nrhs,
        NAT) complex64, lam or None, itno, tole)."""
        p, src, adia, dadia = (np.ascontiguousarray(a, dtype=np.complex64) for a in (p, src, adia, dadia))
        nrhs = p.shape[0]
        grad = np.zeros((nrhs, self.nat), dtype=np.complex64)
        lam = np.zeros_like(p) if want_lam else None
        it = np.zeros(nrhs, dtype=np.int32)
        tole = np.zeros(nrhs, dtype=np.float32)
        rc = self.lib.ddscat_b200_adjoint_f32(nrhs, _ptr(p), _ptr(src), _ptr(adia), _ptr(dadia), maxit, tol,
                                              _ptr(grad), _ptr(lam), _ptr(it), _ptr(tole))
        self._check("adjoint", rc)
        return grad, lam, it, tole

    def adjoint_fwd(self, e, src, adia, dadia, maxit=1000, tol=1e-5, want_p=False):
        """Per-site derivatives of s_k^T P with the forward solution P of A P = e
        recomputed inside the call (ddscat_b200_adjoint_fwd_f32).  e, adia,
        dadia: (3*NAT,) complex64; src: (nsrc, 3*NAT) complex64; NumPy arrays
        or CUDA tensors (all of one kind).  Returns (grad (nsrc, NAT), p or None,
        itno, tole) with itno / tole of the forward solve first."""
        dev = hasattr(e, "data_ptr")
        if not dev:
            e, adia, dadia = (np.ascontiguousarray(a, dtype=np.complex64).reshape(-1) for a in (e, adia, dadia))
            src = np.ascontiguousarray(src, dtype=np.complex64).reshape(-1, 3 * self.nat)
        nsrc = int(src.shape[0])
        if dev:
            import torch

            grad = torch.zeros((nsrc, self.nat), dtype=torch.complex64, device=e.device)
            p = torch.zeros(3 * self.nat, dtype=torch.complex64, device=e.device) if want_p else None
        else:
            grad = np.zeros((nsrc, self.nat), dtype=np.complex64)
            p = np.zeros(3 * self.nat, dtype=np.complex64) if want_p else None
        it = np.zeros(nsrc + 1, dtype=np.int32)
        tole = np.zeros(nsrc + 1, dtype=np.float32)
        rc = self.lib.ddscat_b200_adjoint_fwd_f32(nsrc, _vptr(e), _vptr(src), _vptr(adia), _vptr(dadia), maxit, tol,
                                                  _vptr(grad), _vptr(p), _ptr(it), _ptr(tole))
        self._check("adjoint_fwd", rc)
        return grad, p, it, tole

    def ffweights(self, aks, ems, x0, e02=1.0, out=None):
        """Far-field adjoint sources (nw, 3*NAT) complex64 built on the GPU
        (ddscat_b200_ffweights_f32): w_k^T P is SCAT's amplitude along ems[k]
        at scattering wave vector aks[k].  out: optional CUDA tensor or NumPy
        array to fill; a NumPy array is returned when none is given."""
        aksd = np.ascontiguousarray(aks, dtype=np.float64).reshape(-1, 3)
        emd = np.ascontiguousarray(ems, dtype=np.float64).reshape(-1, 3)
        x0d = np.ascontiguousarray(x0, dtype=np.float64)
        nw = aksd.shape[0]
        if out is None:
            out = np.zeros((nw, 3 * self.nat), dtype=np.complex64)
        rc = self.lib.ddscat_b200_ffweights_f32(nw, _ptr(aksd), _ptr(emd), _ptr(x0d), float(e02), _vptr(out))
        self._check("ffweights", rc)
        return out

    def multi_solve(self, targets_, name="qmrccg", maxit=1000, tol=1e-5, replace=True, symmetric=True, nthreads=0,
                    check=True, autotune=False, graph=False):
        """Solve many targets of uneven size together.  targets_: list of dicts
        with dims (nx, ny, nz), iocc (NAT int16), ak (3,), b, x, adia
        ((nrhs, 3*NAT) complex64 host arrays; x in/out).  Returns BatchOut over
        all RHS in target order."""
        nt = len(targets_)
        dims = np.ascontiguousarray([t["dims"] for t in targets_], dtype=np.int32).reshape(-1)
        occs = [np.ascontiguousarray(t["iocc"], dtype=np.int16) for t in targets_]
        aks = np.ascontiguousarray([t["ak"] for t in targets_], dtype=np.float32).reshape(-1)
        nr = np.ascontiguousarray([t["b"].shape[0] for t in targets_], dtype=np.int32)
        for t in targets_:
            for key in ("b", "x", "adia"):
                a = t[key]
                if a.dtype != np.complex64 or not a.flags.c_contiguous:
                    raise ValueError(f"{key} must be a C-contiguous complex64 array")
        P = ct.c_void_p * nt
        po = P(*[a.ctypes.data for a in occs])
        pb = P(*[t["b"].ctypes.data for t in targets_])
        px = P(*[t["x"].ctypes.data for t in targets_])
        pa = P(*[t["adia"].ctypes.data for t in targets_])
        total = int(nr.sum())
        it = np.zeros(total, dtype=np.int32)
        tole = np.zeros(total, dtype=np.float32)
        nc = np.zeros(total, dtype=np.int32)
        st = np.zeros(total, dtype=np.int32)
        code = BATCH_SOLVERS[name] | (REPLACE_RESIDUAL if replace else 0) | (QMR_SYMMETRIC if symmetric else 0)
        code |= AUTOTUNE if autotune else 0
        code |= GRAPH if graph else 0
        rc = self.lib.ddscat_b200_multi_solve_f32(nt, _ptr(dims), ct.cast(po, ct.c_void_p), _ptr(aks), _ptr(nr),
                                                  ct.cast(pb, ct.c_void_p), ct.cast(px, ct.c_void_p),
                                                  ct.cast(pa, ct.c_void_p), code, maxit, tol, nthreads, _ptr(it),
                                                  _ptr(tole), _ptr(nc), _ptr(st))
        if check:
            self._check("multi_solve", rc)
        return BatchOut(rc, it, tole, nc, st)

    def last_solve_stats(self):
        ms, rhs, calls = ct.c_double(), ct.c_longlong(), _I()
        self.lib.ddscat_b200_last_solve_stats(ct.byref(ms), ct.byref(rhs), ct.byref(calls))
        return ms.value, rhs.value, calls.value

    def residual_f64(self, b, x, adia, aoff=None):
        nrhs = int(b.shape[0])
        out = np.zeros(nrhs, dtype=np.float64)
        rc = self.lib.ddscat_b200_residual_f64(nrhs, _vptr(b), _vptr(x), _vptr(adia), _vptr(aoff),
                                               out.ctypes.data_as(_D))
        self._check("residual_f64", rc)
        return out

    def matvec_ms(self, nrhs=1, iters=10, cwhat="N"):
        ms = _F(0.0)
        self._check("matvec_timing", self.lib.ddscat_b200_matvec_timing(nrhs, iters, ord(cwhat), ct.byref(ms)))
        return ms.value

    def make_inputs(self, ks, es, x0, m, icomp=None, b=None, adia=None, cmdpol="LATTDR"):
        """b and CXADIA (nrhs, 3*NAT) for wave vectors ks (nrhs, 3) and
        polarisations es (nrhs, 3) on the GPU.  m: refractive index or list of
        them; icomp: NAT material indices (1-based, 0 vacuum) or None; cmdpol:
        the polarisability prescription, "LATTDR", "GKDLDR" or "FLTRCD".  b / adia:
        optional preallocated outputs (NumPy arrays or CUDA tensors); NumPy
        arrays are returned when none are given."""
        kf = np.ascontiguousarray(ks, dtype=np.float32).reshape(-1, 3)
        nrhs = kf.shape[0]
        ef = _c64(es, 3 * nrhs)
        x0f = np.ascontiguousarray(x0, dtype=np.float32)
        mf = _c64(np.atleast_1d(m))
        ic = None if icomp is None else np.ascontiguousarray(icomp, dtype=np.int16)
        if b is None and adia is None:
            b = np.zeros((nrhs, 3 * self.nat), dtype=np.complex64)
            adia = np.zeros_like(b)
        pol = CMDPOL[cmdpol]
        if pol == CMDPOL["LATTDR"]:
            rc = self.lib.ddscat_b200_make_inputs_f32(nrhs, _ptr(kf), _ptr(ef), _ptr(x0f), int(mf.size), _ptr(mf),
                                                      _ptr(ic), _vptr(b), _vptr(adia))
        else:
            rc = self.lib.ddscat_b200_make_inputs_pol_f32(pol, nrhs, _ptr(kf), _ptr(ef), _ptr(x0f), int(mf.size),
                                                          _ptr(mf), _ptr(ic), _vptr(b), _vptr(adia))
        self._check("make_inputs", rc)
        return b, adia

    def mueller(self, ak, e01, e02, em2, f11, f21, f12, f22):
        """(S1..S4 per direction (ndir, 4) complex64, Mueller S_ij (ndir, 4, 4)) from
        the f1/f2 outputs of scat() for the two incident polarisations."""
        f = [_c64(v) for v in (f11, f21, f12, f22)]
        ndir = f[0].size
        akf = np.ascontiguousarray(ak, dtype=np.float32)
        e1, e2 = _c64(e01, 3), _c64(e02, 3)
        em2f = np.ascontiguousarray(em2, dtype=np.float32).reshape(ndir, 3)
        s = np.zeros((ndir, 4), dtype=np.complex64)
        m = np.zeros((ndir, 4, 4), dtype=np.float64)
        rc = self.lib.ddscat_b200_mueller_f32(ndir, _ptr(akf), _ptr(e1), _ptr(e2), _ptr(em2f), *[_ptr(v) for v in f],
                                              _ptr(s), m.ctypes.data_as(_D))
        self._check("mueller", rc)
        return s, m

    def mueller_f64(self, ak, e01, e02, em2, f11, f21, f12, f22):
        """mueller() with complex-double amplitudes (e.g. from scat_amplitudes_f64):
        (S1..S4 (ndir, 4) complex128, S_ij (ndir, 4, 4))."""
        f = [np.ascontiguousarray(v, dtype=np.complex128) for v in (f11, f21, f12, f22)]
        ndir = f[0].size
        akd = np.ascontiguousarray(ak, dtype=np.float64)
        e1 = np.ascontiguousarray(e01, dtype=np.complex128)
        e2 = np.ascontiguousarray(e02, dtype=np.complex128)
        em2d = np.ascontiguousarray(em2, dtype=np.float64).reshape(ndir, 3)
        s = np.zeros((ndir, 4), dtype=np.complex128)
        m = np.zeros((ndir, 4, 4), dtype=np.float64)
        rc = self.lib.ddscat_b200_mueller_f64(ndir, _ptr(akd), _ptr(e1), _ptr(e2), _ptr(em2d),
                                              *[_ptr(v) for v in f], _ptr(s), m.ctypes.data_as(_D))
        self._check("mueller_f64", rc)
        return s, m

    def scat_amplitudes_f64(self, x, ak, aks, em1, em2, x0, dx=(1.0, 1.0, 1.0), e02=1.0):
        """All-FP64 scattering amplitudes (f1, f2), each (nrhs, ndir) complex128,
        of the polarisations x ((nrhs, 3*NAT) complex128, NumPy or CUDA tensor),
        normalised like the f1/f2 of scat()."""
        nrhs = int(x.shape[0])
        if not hasattr(x, "data_ptr") and (x.dtype != np.complex128 or not x.flags.c_contiguous):
            raise ValueError("x must be a C-contiguous complex128 array")
        aksd = np.ascontiguousarray(aks, dtype=np.float64).reshape(-1, 3)
        ndir = aksd.shape[0]
        em1d = np.ascontiguousarray(em1, dtype=np.float64).reshape(ndir, 3)
        em2d = np.ascontiguousarray(em2, dtype=np.float64).reshape(ndir, 3)
        akd = np.ascontiguousarray(ak, dtype=np.float64)
        dxd = np.ascontiguousarray(dx, dtype=np.float64)
        x0d = np.ascontiguousarray(x0, dtype=np.float64)
        f1 = np.zeros((nrhs, ndir), dtype=np.complex128)
        f2 = np.zeros((nrhs, ndir), dtype=np.complex128)
        rc = self.lib.ddscat_b200_scat_amplitudes_f64(nrhs, _vptr(x), ndir, _ptr(akd), _ptr(aksd), _ptr(em1d),
                                                      _ptr(em2d), _ptr(dxd), _ptr(x0d), float(e02), _ptr(f1),
                                                      _ptr(f2))
        self._check("scat_amplitudes_f64", rc)
        return f1, f2

    def scat_csca_f64(self, x, ak, e01, x0, dx=(1.0, 1.0, 1.0), etasca=0.5, e02=1.0):
        """All-FP64 Csca, Csca*g, Csca*<cos^2>, backscatter and NAVG of the
        polarisations x ((nrhs, 3*NAT) complex128, NumPy or CUDA tensor) over
        SCAT's integration directions for incident polarisations e01 ((nrhs, 3)
        or (3,)): the FP64 counterpart of scat()'s cross sections."""
        nrhs = int(x.shape[0])
        if not hasattr(x, "data_ptr") and (x.dtype != np.complex128 or not x.flags.c_contiguous):
            raise ValueError("x must be a C-contiguous complex128 array")
        e01c = np.ascontiguousarray(np.broadcast_to(np.asarray(e01, dtype=np.complex64).reshape(-1, 3), (nrhs, 3)))
        akf = np.ascontiguousarray(ak, dtype=np.float32)
        dxf = np.ascontiguousarray(dx, dtype=np.float32)
        x0f = np.ascontiguousarray(x0, dtype=np.float32)
        cb, cs, cg2 = (np.zeros(nrhs) for _ in range(3))
        cg = np.zeros((nrhs, 3))
        navg = np.zeros(nrhs, dtype=np.int32)
        rc = self.lib.ddscat_b200_scat_csca_f64(nrhs, _vptr(x), _ptr(akf), _ptr(e01c), float(etasca), _ptr(dxf),
                                                _ptr(x0f), float(e02), _ptr(cb), _ptr(cs), _ptr(cg), _ptr(cg2),
                                                _ptr(navg))
        self._check("scat_csca_f64", rc)
        return {"cbksca": cb, "csca": cs, "cscag": cg, "cscag2": cg2, "navg": navg}

    def autotune(self, iters=5):
        """Tune the prepared target's FFT launch shapes; returns (default ms, best ms) per MATVEC."""
        d, b = _F(0.0), _F(0.0)
        self._check("autotune", self.lib.ddscat_b200_autotune_f32(iters, ct.byref(d), ct.byref(b)))
        return d.value, b.value

    def launch_count(self):
        return int(self.lib.ddscat_b200_launch_count())

    def release(self):
        return self.lib.ddscat_cuda_release()
