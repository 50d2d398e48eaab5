"""The drop-in boundary through DDSCAT's own loader, on CPU.

oracle/_ref/ddscat_bridge_driver links the reference's C loader
(ddscat_cuda_unified/cuda/ddscat_cuda_loader.c, compiled unmodified by
oracle/Makefile) with a C stand-in for the Fortran bridge.  Its `probe` mode
makes one ddscat_cuda_loader_prepare_green_f32 call against the library named
by DDSCAT_CUDA_DLL and prints the status.  Checked here: the loader's own
codes for stand-in libraries (1001 no library, 1002 a mandatory symbol
missing, -777 no prepare_green, loader.c:88-101), and that both of this
project's libraries pass the loader's 14 mandatory dlsym lookups (the status
is then the library's own: without a GPU its prepare fails with a CUDA
error, never a loader code)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ddscat_bridge_driver")
STUB = os.path.join(ROOT, "tests", "loader_stub.c")
LIBS = [os.path.join(ROOT, "ddscat-cuda_b200", "lib", n)
        for n in ("libddscat_matvec_cuda.so", "libddscat_matvec_cuda_slice.so")]

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER) or shutil.which("gcc") is None,
                                reason="bridge driver (oracle/Makefile) or gcc not available")


def _probe(lib):
    env = dict(os.environ, DDSCAT_CUDA_DLL=lib, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([DRIVER, "probe"], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    return int(out.stdout.strip().splitlines()[-1]), out


def _stub(tmp_path, omit=None):
    so = tmp_path / f"stub_{omit or 'full'}.so"
    cmd = ["gcc", "-shared", "-fPIC", "-fvisibility=hidden", "-o", str(so), STUB]
    if omit:
        cmd.insert(1, f"-DOMIT_{omit}")
    subprocess.run(cmd, check=True)
    return str(so)


def test_loader_accepts_complete_stub(tmp_path):
    rc, out = _probe(_stub(tmp_path))
    assert rc == 0
    assert "DDSCAT CUDA library loaded" in out.stdout


@pytest.mark.parametrize("omit", ["PREPARE", "APPLY", "QMRCCG", "SCAT"])
def test_loader_reports_missing_mandatory_symbol(tmp_path, omit):
    rc, _ = _probe(_stub(tmp_path, omit))
    assert rc == 1002


def test_loader_reports_missing_prepare_green(tmp_path):
    rc, _ = _probe(_stub(tmp_path, "PREPARE_GREEN"))
    assert rc == -777


def test_loader_reports_missing_library(tmp_path):
    rc, _ = _probe(str(tmp_path / "no_such_library.so"))
    assert rc == 1001


@pytest.mark.parametrize("lib", LIBS, ids=["fft3d", "slices"])
def test_loader_resolves_every_entry_point_of_this_library(lib):
    if not os.path.exists(lib):
        pytest.skip("library not built")
    rc, out = _probe(lib)
    assert rc not in (1001, 1002, -777), out.stderr
    assert "DDSCAT CUDA library loaded" in out.stdout
