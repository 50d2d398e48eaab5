"""CPU tests of the C-ABI boundary: both layout libraries load, export every
symbol the headers in include/ declare, and reject bad arguments with the
reference's codes before touching the GPU (no compute calls here)."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

import ddscat_b200 as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in ("ddscat_matvec_cuda.h", "ddscat_b200.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"DDSCAT_CUDA_API\s+[^;(]*?\b(ddscat_\w+)\s*\(", txt)
    return names


def test_headers_declare_reference_abi():
    names = _declared()
    assert len(names) == len(set(names))
    for s in D.SOLVERS:
        assert f"ddscat_cuda_solve_{s}_f32" in names
    ref15 = [n for n in names if n.startswith("ddscat_cuda_")]
    assert len(ref15) == 15
    assert set(names) == set(D.EXPORTS)


@pytest.mark.parametrize("layout", ["fft3d", "slices"])
def test_library_exports_every_declared_symbol(layout):
    lib = D.load(layout)
    for name in _declared():
        assert hasattr(lib, name), name
    assert lib.ddscat_b200_layout() == (1 if layout == "slices" else 0)


def test_loader_lookup_names():
    # the reference loader dlopens these names (ddscat_cuda_loader.c:45-50)
    assert os.path.basename(D.lib_path("fft3d")) == "libddscat_matvec_cuda.so"
    assert os.path.basename(D.lib_path("slices")) == "libddscat_matvec_cuda_slice.so"


def test_argument_errors_before_prepare():
    lib = D.load("fft3d")
    assert lib.ddscat_cuda_release() == 0
    x = np.zeros(3, dtype=np.complex64)
    assert lib.ddscat_cuda_apply_f32(ord("N"), x.ctypes.data, x.ctypes.data, x.ctypes.data, x.ctypes.data) == 10
    assert b"not prepared" in lib.ddscat_cuda_last_error()
    it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
    codes = {"gpbicg": 30, "qmrccg": 50, "pbcgst": 70, "pbcgs2": 90, "petrkp": 110, "bicgstab4": 130,
             "gpbicgstab2": 150, "gpbicgstab4": 180}
    for s, code in codes.items():
        f = getattr(lib, f"ddscat_cuda_solve_{s}_f32")
        rc = f(x.ctypes.data, x.ctypes.data, x.ctypes.data, x.ctypes.data, 3, 10, 1e-5, ct.byref(it), ct.byref(tole),
               ct.byref(nc))
        assert rc == code, s
    occ = np.ones(8, dtype=np.int16)
    # nat0 > nat, bad ipbc, bad idipint, NAT != NX*NY*NZ
    assert lib.ddscat_cuda_prepare_green_f32(2, 2, 2, 0, 8, 9, 0, 0, 0, 0, 1, 0, 0, 1, 1, 1, occ.ctypes.data) == 201
    assert lib.ddscat_cuda_prepare_green_f32(2, 2, 2, 2, 8, 8, 0, 0, 0, 0, 1, 0, 0, 1, 1, 1, occ.ctypes.data) == 201
    assert lib.ddscat_cuda_prepare_green_f32(2, 2, 2, 0, 8, 8, 3, 0, 0, 0, 1, 0, 0, 1, 1, 1, occ.ctypes.data) == 201
    assert lib.ddscat_cuda_prepare_green_f32(2, 2, 2, 0, 9, 8, 0, 0, 0, 0, 1, 0, 0, 1, 1, 1, occ.ctypes.data) == 201
    assert lib.ddscat_cuda_prepare_green_f32(2, 2, 2, 1, 8, 8, 0, 0, 0, 0, 1, 0, 0, 1, 1, 1, occ.ctypes.data) == 202
    assert lib.ddscat_cuda_prepare_f32(2, 2, 2, 0, 8, 8, None, occ.ctypes.data) == 1
    cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
    assert lib.ddscat_cuda_evalq_f32(1, None, None, None, None, 1.0, 0.0, 0.0, 1.0, ct.byref(cabs), ct.byref(cext),
                                     ct.byref(cpha)) == 300
