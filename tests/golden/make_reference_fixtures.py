"""Generate golden fixtures by running the REFERENCE library on a B200.

The reference backend (ddscat_cuda_unified/cuda/ddscat_matvec_cuda.cu) is built
unmodified by oracle/Makefile into oracle/_ref/.  This script calls it through
its own C ABI on small seeded inputs and stores inputs and outputs in
tests/golden/reference_fixtures.npz.  tests/test_oracle_pinned.py then checks
the CPU oracle against these outputs (no GPU needed), which pins the oracle to
the reference's actual behaviour.

A second set at configuration size (reference_fixtures_c1.npz): the whole
small-sphere workload (32^3 sphere, m = 1.50+0.01i, x = 5, PBCGS2 at tol 1e-5
for both polarisations, EVALQ, SCAT at ETASCA 0.5 with f1/f2 on 0..180 deg at
1 deg in two scattering planes) and a 64^3 MATVEC ('N' and 'C').  Its inputs
are regenerated from seeds by c1_problem() and mv64_inputs() below, so only
outputs are stored (the 64^3 MATVEC as seeded samples and projections).

A third set (reference_fixtures_edge.npz) holds the edge cases of
edge_cases.py: every solver with a nonzero CXAOFF, the single-site target
(PBCGS2 and QMRCCG return codes) and the MATVEC of hollow targets with vacant
rows and planes.

A fourth set (reference_fixtures_pbc.npz) holds periodic targets (IPBC = 1,
the replica-sum Green tensor of cu:634-643 and the full-tensor MATVEC branch of
cu:113): MATVECs for periodicity in y (JPBC 1), in z (JPBC 2) and in y and z
(JPBC 3), one with IDIPINT = 1, one on a caller-supplied full-grid spectrum
(prepare_f32 with IPBC = 1), and a PBCGS2 solve with EVALQ and SCAT's
selected-direction amplitudes on a target periodic in y and z (the cases of
edge_cases.pbc_cases and edge_cases.pbc_solve_problem).

A fifth set (reference_fixtures_dx.npz) holds rectangular lattices (dx1..dx3 =
1.0, 0.9, 1.1): MATVECs with IDIPINT 0 and 1 and a periodic one, and a QMRCCG
solve with EVALQ and SCAT (edge_cases.dx_cases, edge_cases.dx_solve_problem).

A sixth set (reference_fixtures_limits.npz) holds the limit cases of all eight
solvers (edge_cases.limits_problem): MAXIT reached, a zero right-hand side and
a nonzero initial guess, with return codes, ITNO, TOLE, NCOMPTE and x.

Run on a GPU machine:  python tests/golden/make_reference_fixtures.py [base|c1|edge|pbc|dx|limits|all]
"""
import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "ddscat-cuda_b200"))

from ddscat_b200 import targets  # noqa: E402
import ddscat_b200 as D  # noqa: E402
from oracle import ddscat_oracle as O  # noqa: E402

sys.path.insert(0, HERE)
import edge_cases as EC  # noqa: E402

OUT = os.path.join(HERE, "reference_fixtures.npz")
OUT_C1 = os.path.join(HERE, "reference_fixtures_c1.npz")
OUT_EDGE = os.path.join(HERE, "reference_fixtures_edge.npz")
OUT_PBC = os.path.join(HERE, "reference_fixtures_pbc.npz")
OUT_DX = os.path.join(HERE, "reference_fixtures_dx.npz")
OUT_LIM = os.path.join(HERE, "reference_fixtures_limits.npz")
C1_TOL, C1_MAXIT, C1_ETASCA = 1e-5, 500, 0.5
MV64_SAMPLES, MV64_PROJ = 8192, 4


def c1_problem():
    """The small-sphere workload: 32^3 sphere, m = 1.50+0.01i, x = 5, one
    orientation, polarisations e01 = y and e02 = z (seeded, deterministic)."""
    return targets.make_problem(32, m=1.5 + 0.01j, x=5.0)


def c1_directions(prob, r):
    """SCAT's selected directions for RHS r: theta 0..180 deg at 1 deg in the
    phi = 0 and 90 deg planes (362 directions), float32 AKS, EM1, EM2."""
    k = prob.incid[r].k
    aks, em1, em2 = targets.scattering_planes(k, prob.incid[r].e)
    return aks.astype(np.float32), em1.astype(np.float32), em2.astype(np.float32)


def mv64_inputs():
    """A 64^3 MATVEC case from seed 64: 70 % random occupancy, random x (zero
    on vacuum sites), CXADIA and CXAOFF, k of modulus ~0.7; and the sample
    indices and projection vectors its output is stored as."""
    rng = np.random.default_rng(64)
    n = 64
    nat = n ** 3
    iocc = (rng.random(nat) < 0.7).astype(np.int16)
    ak = (rng.normal(size=3) * 0.4).astype(np.float32)
    c = lambda s=1.0: (s * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)  # noqa: E731
    x, adia, aoff = c(), c(), c(0.3)
    x[np.tile(iocc == 0, 3)] = 0
    idx = np.sort(rng.choice(3 * nat, MV64_SAMPLES, replace=False))
    proj = (rng.normal(size=(MV64_PROJ, 3 * nat)) + 1j * rng.normal(size=(MV64_PROJ, 3 * nat))) / np.sqrt(3 * nat)
    return (n, n, n), iocc, ak, x, adia, aoff, idx, proj


def mv64_summary(y, idx, proj):
    """What the 64^3 MATVEC output is stored as: seeded samples, the L2 norm and
    projections onto seeded random vectors (complex128)."""
    y = np.asarray(y)
    return y[idx], np.array([np.linalg.norm(y.astype(np.complex128))]), proj @ y.astype(np.complex128)


def ref_lib(layout="fft3d"):
    path = os.path.join(ROOT, "oracle", "_ref", f"libddscat_ref_{layout}.so")
    lib = ct.CDLL(path, mode=ct.RTLD_LOCAL)
    _declare_ref(lib)  # the reference exports the same 15 names and signatures
    return lib


def _declare_ref(lib):
    _P, _I, _F = ct.c_void_p, ct.c_int, ct.c_float
    _D = ct.POINTER(ct.c_double)
    lib.ddscat_cuda_prepare_green_f32.argtypes = [_I] * 7 + [_F] * 9 + [_P]
    lib.ddscat_cuda_prepare_f32.argtypes = [_I] * 6 + [_P, _P]
    lib.ddscat_cuda_apply_f32.argtypes = [_I, _P, _P, _P, _P]
    for s in D.SOLVERS:
        getattr(lib, f"ddscat_cuda_solve_{s}_f32").argtypes = [_P, _P, _P, _P, _I, _I, _F, ct.POINTER(_I),
                                                                ct.POINTER(_F), ct.POINTER(_I)]
    lib.ddscat_cuda_evalq_f32.argtypes = [_I, _P, _P, _P, _P, _F, _F, _F, _F, _D, _D, _D]
    lib.ddscat_cuda_scat_f32.argtypes = [_I, _I, _P, _P, _P, _P, _P, _F, _F, _P, _P, _D, _D, _D, _D, ct.POINTER(_I),
                                         _P, _P]
    lib.ddscat_cuda_last_error.restype = ct.c_char_p


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


def main():
    lib = ref_lib("fft3d")
    fx = {}
    # ---- A: MATVEC on a random 7x6x5 grid (prepare_green, both CWHAT), IDIPINT 0 and 1
    rng = np.random.default_rng(20261203)
    for idip in (0, 1):
        nx, ny, nz = 7, 6, 5
        nat = nx * ny * nz
        iocc = (rng.random(nat) < 0.75).astype(np.int16)
        ak = (rng.normal(size=3) * 0.4).astype(np.float32)
        x = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
        x[np.tile(iocc == 0, 3)] = 0  # DDSCAT passes zeros on vacuum sites
        adia = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
        aoff = (0.3 * (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat))).astype(np.complex64)
        rc = lib.ddscat_cuda_prepare_green_f32(nx, ny, nz, 0, nat, int(iocc.sum()), idip, 0.0, 0.0, 0.0, *map(float, ak), 1.0,
                                               1.0, 1.0, _p(iocc))
        assert rc == 0, lib.ddscat_cuda_last_error()
        for cw in "NC":
            y = np.empty_like(x)
            assert lib.ddscat_cuda_apply_f32(ord(cw), _p(x), _p(y), _p(adia), _p(aoff)) == 0
            fx[f"A{idip}_y{cw}"] = y
        fx.update({f"A{idip}_dims": np.array([nx, ny, nz]), f"A{idip}_iocc": iocc, f"A{idip}_ak": ak,
                   f"A{idip}_x": x, f"A{idip}_adia": adia, f"A{idip}_aoff": aoff})
    # ---- B: 12^3 sphere, LDR, all eight solvers + EVALQ + SCAT
    n = 12
    prob = targets.make_problem(n, m=1.5 + 0.01j, x=2.0)
    k = prob.incid[0].k.astype(np.float32)
    iocc = prob.iocc
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    rc = lib.ddscat_cuda_prepare_green_f32(n, n, n, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0, *map(float, k), 1.0, 1.0, 1.0,
                                           _p(iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    fx.update({"B_n": np.array([n]), "B_iocc": iocc, "B_k": k, "B_b": b, "B_adia": adia, "B_aoff": aoff,
               "B_e": prob.incid[0].e.astype(np.complex64), "B_x0": np.array(prob.x0, dtype=np.float32)})
    for s in D.SOLVERS:
        xs = np.zeros_like(b)
        it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
        rc = getattr(lib, f"ddscat_cuda_solve_{s}_f32")(_p(b), _p(xs), _p(adia), _p(aoff), b.size, 300, 1e-5,
                                                        ct.byref(it), ct.byref(tole), ct.byref(nc))
        fx[f"B_{s}_rc"] = np.array([rc])
        fx[f"B_{s}_x"] = xs
        fx[f"B_{s}_meta"] = np.array([it.value, tole.value, nc.value], dtype=np.float64)
        if s == "qmrccg":
            cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
            assert lib.ddscat_cuda_evalq_f32(1, None, None, None, None, *map(float, k), 1.0, ct.byref(cabs), ct.byref(cext),
                                             ct.byref(cpha)) == 0
            fx["B_evalq"] = np.array([cabs.value, cext.value, cpha.value])
            th = np.deg2rad(np.arange(0.0, 181.0, 30.0))
            kk = float(np.linalg.norm(k))
            aks = np.array([[kk * np.cos(t), kk * np.sin(t), 0.0] for t in th], dtype=np.float32)
            em1 = np.array([[-np.sin(t), np.cos(t), 0.0] for t in th], dtype=np.float32)
            em2 = np.array([[0.0, 0.0, 1.0] for t in th], dtype=np.float32)
            dx = np.ones(3, dtype=np.float32)
            x0 = np.array(prob.x0, dtype=np.float32)
            e01 = prob.incid[0].e.astype(np.complex64)
            f1 = np.zeros(len(th), dtype=np.complex64)
            f2 = np.zeros(len(th), dtype=np.complex64)
            cb, cs, cg2 = ct.c_double(), ct.c_double(), ct.c_double()
            cg = (ct.c_double * 3)()
            navg = ct.c_int()
            rc = lib.ddscat_cuda_scat_f32(0, len(th), _p(k), _p(aks), _p(dx), _p(em1), _p(em2), 1.0, 3.0, _p(e01),
                                          _p(x0), ct.byref(cb), ct.byref(cs), ct.cast(cg, ct.POINTER(ct.c_double)),
                                          ct.byref(cg2), ct.byref(navg), _p(f1), _p(f2))
            assert rc == 0, lib.ddscat_cuda_last_error()
            fx["B_scat"] = np.array([cb.value, cs.value, cg[0], cg[1], cg[2], cg2.value, navg.value])
            fx.update({"B_aks": aks, "B_em1": em1, "B_em2": em2, "B_f1": f1, "B_f2": f2})
    lib.ddscat_cuda_release()
    # ---- C: prepare_f32 with a CPU-supplied octant (FP64 oracle octant rounded to c64)
    nx, ny, nz = 6, 5, 4
    nat = nx * ny * nz
    iocc = np.ones(nat, dtype=np.int16)
    gp = O.GreenParams(nx, ny, nz, ak=(0.3, -0.2, 0.5))
    oct6 = O.green_octant(gp).astype(np.complex64)
    x = (rng.normal(size=3 * nat) + 1j * rng.normal(size=3 * nat)).astype(np.complex64)
    adia = np.full(3 * nat, 1.7 - 0.4j, dtype=np.complex64)
    aoff = np.zeros(3 * nat, dtype=np.complex64)
    assert lib.ddscat_cuda_prepare_f32(nx, ny, nz, 0, nat, nat, _p(oct6), _p(iocc)) == 0
    y = np.empty_like(x)
    assert lib.ddscat_cuda_apply_f32(ord("N"), _p(x), _p(y), _p(adia), _p(aoff)) == 0
    fx.update({"C_dims": np.array([nx, ny, nz]), "C_oct": oct6, "C_x": x, "C_adia": adia, "C_y": y})
    lib.ddscat_cuda_release()
    np.savez_compressed(OUT, **fx)
    print("wrote", OUT, len(fx), "arrays")


def main_c1():
    lib = ref_lib("fft3d")
    fx = {}
    # ---- 64^3 MATVEC, both CWHAT
    dims, iocc, ak, x, adia, aoff, idx, proj = mv64_inputs()
    nat = int(np.prod(dims))
    rc = lib.ddscat_cuda_prepare_green_f32(*dims, 0, nat, int(iocc.sum()), 0, 0.0, 0.0, 0.0, *map(float, ak), 1.0, 1.0,
                                           1.0, _p(iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    for cw in "NC":
        y = np.empty_like(x)
        assert lib.ddscat_cuda_apply_f32(ord(cw), _p(x), _p(y), _p(adia), _p(aoff)) == 0
        smp, nrm, prj = mv64_summary(y, idx, proj)
        fx.update({f"M64_{cw}_samples": smp, f"M64_{cw}_norm": nrm, f"M64_{cw}_proj": prj})
    lib.ddscat_cuda_release()
    # ---- the small-sphere workload, PBCGS2 per polarisation, EVALQ, SCAT
    prob = c1_problem()
    k = prob.incid[0].k.astype(np.float32)
    rc = lib.ddscat_cuda_prepare_green_f32(32, 32, 32, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0, *map(float, k), 1.0,
                                           1.0, 1.0, _p(prob.iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    aoff = prob.aoff()
    dx = np.ones(3, dtype=np.float32)
    x0 = np.array(prob.x0, dtype=np.float32)
    for r in range(len(prob.incid)):
        b, adia = prob.rhs(r), prob.adia(r)
        xs = np.zeros_like(b)
        it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
        rc = lib.ddscat_cuda_solve_pbcgs2_f32(_p(b), _p(xs), _p(adia), _p(aoff), b.size, C1_MAXIT, C1_TOL,
                                              ct.byref(it), ct.byref(tole), ct.byref(nc))
        assert rc == 0, lib.ddscat_cuda_last_error()
        fx[f"C1_{r}_x"] = np.concatenate([xs[c * prob.nat:(c + 1) * prob.nat][prob.occ] for c in range(3)])
        fx[f"C1_{r}_meta"] = np.array([it.value, tole.value, nc.value], dtype=np.float64)
        fx[f"C1_{r}_inputs"] = np.array([b.astype(np.complex128).sum(), adia.astype(np.complex128).sum()])
        cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
        assert lib.ddscat_cuda_evalq_f32(1, None, None, None, None, *map(float, k), 1.0, ct.byref(cabs),
                                         ct.byref(cext), ct.byref(cpha)) == 0
        fx[f"C1_{r}_evalq"] = np.array([cabs.value, cext.value, cpha.value])
        aks, em1, em2 = c1_directions(prob, r)
        e01 = prob.incid[r].e.astype(np.complex64)
        f1 = np.zeros(len(aks), dtype=np.complex64)
        f2 = np.zeros(len(aks), dtype=np.complex64)
        cb, cs, cg2 = ct.c_double(), ct.c_double(), ct.c_double()
        cg = (ct.c_double * 3)()
        navg = ct.c_int()
        rc = lib.ddscat_cuda_scat_f32(0, len(aks), _p(k), _p(aks), _p(dx), _p(em1), _p(em2), 1.0, C1_ETASCA,
                                      _p(e01), _p(x0), ct.byref(cb), ct.byref(cs),
                                      ct.cast(cg, ct.POINTER(ct.c_double)), ct.byref(cg2), ct.byref(navg), _p(f1),
                                      _p(f2))
        assert rc == 0, lib.ddscat_cuda_last_error()
        fx[f"C1_{r}_scat"] = np.array([cb.value, cs.value, cg[0], cg[1], cg[2], cg2.value, navg.value])
        fx[f"C1_{r}_f1"] = f1
        fx[f"C1_{r}_f2"] = f2
    lib.ddscat_cuda_release()
    np.savez_compressed(OUT_C1, **fx)
    print("wrote", OUT_C1, len(fx), "arrays")


def _ref_solve(lib, name, b, adia, aoff, maxit, tol):
    xs = np.zeros_like(b)
    it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
    rc = getattr(lib, f"ddscat_cuda_solve_{name}_f32")(_p(b), _p(xs), _p(adia), _p(aoff), b.size, maxit, tol,
                                                       ct.byref(it), ct.byref(tole), ct.byref(nc))
    return rc, xs, np.array([it.value, tole.value, nc.value], dtype=np.float64)


def main_edge():
    lib = ref_lib("fft3d")
    fx = {}
    # ---- nonzero CXAOFF through every solver of edge_cases.SOLVERS_AOFF
    prob, b, adia, aoff = EC.aoff_problem()
    k = prob.incid[0].k.astype(np.float32)
    rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0,
                                           *map(float, k), 1.0, 1.0, 1.0, _p(prob.iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    for s in EC.SOLVERS_AOFF:
        rc, xs, meta = _ref_solve(lib, s, b, adia, aoff, EC.MAXIT, EC.TOL)
        fx[f"O_{s}_rc"] = np.array([rc])
        fx[f"O_{s}_x"] = xs
        fx[f"O_{s}_meta"] = meta
    lib.ddscat_cuda_release()
    # ---- sparse targets: MATVEC ('N', 'C'), PBCGS2 and QMRCCG return codes and meta
    for case in ("single_site",) + EC.HOLLOW:
        prob, b, adia, aoff, x = EC.sparse_problem(case)
        k = prob.incid[0].k.astype(np.float32)
        rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0,
                                               *map(float, k), 1.0, 1.0, 1.0, _p(prob.iocc))
        assert rc == 0, lib.ddscat_cuda_last_error()
        for cw in "NC":
            y = np.empty_like(x)
            assert lib.ddscat_cuda_apply_f32(ord(cw), _p(x), _p(y), _p(adia), _p(aoff)) == 0
            fx[f"S_{case}_y{cw}"] = y
        for s in ("pbcgs2", "qmrccg"):
            rc, xs, meta = _ref_solve(lib, s, b, adia, aoff, 400, EC.TOL)
            fx[f"S_{case}_{s}_rc"] = np.array([rc])
            fx[f"S_{case}_{s}_meta"] = meta
        lib.ddscat_cuda_release()
    np.savez_compressed(OUT_EDGE, **fx)
    print("wrote", OUT_EDGE, len(fx), "arrays")


def main_pbc():
    lib = ref_lib("fft3d")
    fx = {}
    for cs in EC.pbc_cases():
        nx, ny, nz = cs["dims"]
        nat = nx * ny * nz
        rc = lib.ddscat_cuda_prepare_green_f32(nx, ny, nz, 1, nat, int(cs["iocc"].sum()), cs["idipint"], cs["gamma"],
                                               cs["pyd"], cs["pzd"], *map(float, cs["ak"]), 1.0, 1.0, 1.0,
                                               _p(cs["iocc"]))
        assert rc == 0, lib.ddscat_cuda_last_error()
        for cw in "NC":
            y = np.empty_like(cs["x"])
            assert lib.ddscat_cuda_apply_f32(ord(cw), _p(cs["x"]), _p(y), _p(cs["adia"]), _p(cs["aoff"])) == 0
            fx[f"M_{cs['name']}_y{cw}"] = y
        lib.ddscat_cuda_release()
    cs = EC.pbc_cpu_green_case()
    nx, ny, nz = cs["dims"]
    nat = nx * ny * nz
    assert lib.ddscat_cuda_prepare_f32(nx, ny, nz, 1, nat, int(cs["iocc"].sum()), _p(cs["green"]), _p(cs["iocc"])) == 0
    for cw in "NC":
        y = np.empty_like(cs["x"])
        assert lib.ddscat_cuda_apply_f32(ord(cw), _p(cs["x"]), _p(y), _p(cs["adia"]), _p(cs["aoff"])) == 0
        fx[f"M_cpu_y{cw}"] = y
    lib.ddscat_cuda_release()
    prob, gamma, pyd, pzd, aks, em1, em2 = EC.pbc_solve_problem()
    k = prob.incid[0].k.astype(np.float32)
    rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 1, prob.nat, prob.nat0, 0, gamma, pyd, pzd,
                                           *map(float, k), 1.0, 1.0, 1.0, _p(prob.iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    rc, xs, meta = _ref_solve(lib, "pbcgs2", b, adia, aoff, 300, 1e-5)
    fx.update({"P_rc": np.array([rc]), "P_x": xs, "P_meta": meta})
    cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
    assert lib.ddscat_cuda_evalq_f32(1, None, None, None, None, *map(float, k), 1.0, ct.byref(cabs), ct.byref(cext),
                                     ct.byref(cpha)) == 0
    fx["P_evalq"] = np.array([cabs.value, cext.value, cpha.value])
    dx = np.ones(3, dtype=np.float32)
    x0 = np.array(prob.x0, dtype=np.float32)
    f1 = np.zeros(len(aks), dtype=np.complex64)
    f2 = np.zeros(len(aks), dtype=np.complex64)
    cb, csc, cg2 = ct.c_double(), ct.c_double(), ct.c_double()
    cg = (ct.c_double * 3)()
    navg = ct.c_int()
    rc = lib.ddscat_cuda_scat_f32(3, len(aks), _p(k), _p(aks), _p(dx), _p(em1), _p(em2), 1.0, 0.0, None, _p(x0),
                                  ct.byref(cb), ct.byref(csc), ct.cast(cg, ct.POINTER(ct.c_double)), ct.byref(cg2),
                                  ct.byref(navg), _p(f1), _p(f2))
    assert rc == 0, lib.ddscat_cuda_last_error()
    fx.update({"P_scat": np.array([cb.value, csc.value, cg[0], cg[1], cg[2], cg2.value, navg.value]),
               "P_f1": f1, "P_f2": f2})
    lib.ddscat_cuda_release()
    np.savez_compressed(OUT_PBC, **fx)
    print("wrote", OUT_PBC, len(fx), "arrays")


def main_dx():
    lib = ref_lib("fft3d")
    fx = {}
    dx = np.array(EC.DX, dtype=np.float32)
    for cs in EC.dx_cases():
        nx, ny, nz = cs["dims"]
        nat = nx * ny * nz
        rc = lib.ddscat_cuda_prepare_green_f32(nx, ny, nz, cs["ipbc"], nat, int(cs["iocc"].sum()), cs["idipint"],
                                               cs["gamma"], cs["pyd"], 0.0, *map(float, cs["ak"]), *map(float, dx),
                                               _p(cs["iocc"]))
        assert rc == 0, lib.ddscat_cuda_last_error()
        for cw in "NC":
            y = np.empty_like(cs["x"])
            assert lib.ddscat_cuda_apply_f32(ord(cw), _p(cs["x"]), _p(y), _p(cs["adia"]), _p(cs["aoff"])) == 0
            fx[f"M_{cs['name']}_y{cw}"] = y
        lib.ddscat_cuda_release()
    prob, aks, em1, em2 = EC.dx_solve_problem()
    k = prob.incid[0].k.astype(np.float32)
    rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0,
                                           *map(float, k), *map(float, dx), _p(prob.iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    b, adia, aoff = prob.rhs(0), prob.adia(0), prob.aoff()
    rc, xs, meta = _ref_solve(lib, "qmrccg", b, adia, aoff, 300, 1e-5)
    fx.update({"Q_rc": np.array([rc]), "Q_x": xs, "Q_meta": meta})
    cabs, cext, cpha = ct.c_double(), ct.c_double(), ct.c_double()
    assert lib.ddscat_cuda_evalq_f32(1, None, None, None, None, *map(float, k), 1.0, ct.byref(cabs), ct.byref(cext),
                                     ct.byref(cpha)) == 0
    fx["Q_evalq"] = np.array([cabs.value, cext.value, cpha.value])
    x0 = np.array(prob.x0, dtype=np.float32)
    e01 = prob.incid[0].e.astype(np.complex64)
    f1 = np.zeros(len(aks), dtype=np.complex64)
    f2 = np.zeros(len(aks), dtype=np.complex64)
    cb, csc, cg2 = ct.c_double(), ct.c_double(), ct.c_double()
    cg = (ct.c_double * 3)()
    navg = ct.c_int()
    rc = lib.ddscat_cuda_scat_f32(0, len(aks), _p(k), _p(aks), _p(dx), _p(em1), _p(em2), 1.0, 3.0, _p(e01), _p(x0),
                                  ct.byref(cb), ct.byref(csc), ct.cast(cg, ct.POINTER(ct.c_double)), ct.byref(cg2),
                                  ct.byref(navg), _p(f1), _p(f2))
    assert rc == 0, lib.ddscat_cuda_last_error()
    fx.update({"Q_scat": np.array([cb.value, csc.value, cg[0], cg[1], cg[2], cg2.value, navg.value]),
               "Q_f1": f1, "Q_f2": f2})
    lib.ddscat_cuda_release()
    np.savez_compressed(OUT_DX, **fx)
    print("wrote", OUT_DX, len(fx), "arrays")


def main_limits():
    lib = ref_lib("fft3d")
    fx = {}
    prob, b, adia, aoff, x0 = EC.limits_problem()
    k = prob.incid[0].k.astype(np.float32)
    rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0,
                                           *map(float, k), 1.0, 1.0, 1.0, _p(prob.iocc))
    assert rc == 0, lib.ddscat_cuda_last_error()
    zero = np.zeros_like(b)
    for s in D.SOLVERS:
        for tag, bb, xx, maxit, tol in (("maxit", b, zero, 3, 1e-12), ("zero", zero, zero, 10, 1e-5),
                                        ("x0", b, x0, 300, 1e-5)):
            xs = xx.copy()
            it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
            rc = getattr(lib, f"ddscat_cuda_solve_{s}_f32")(_p(bb), _p(xs), _p(adia), _p(aoff), bb.size, maxit, tol,
                                                            ct.byref(it), ct.byref(tole), ct.byref(nc))
            fx[f"L_{s}_{tag}_rc"] = np.array([rc])
            fx[f"L_{s}_{tag}_x"] = xs
            fx[f"L_{s}_{tag}_meta"] = np.array([it.value, tole.value, nc.value], dtype=np.float64)
    lib.ddscat_cuda_release()
    np.savez_compressed(OUT_LIM, **fx)
    print("wrote", OUT_LIM, len(fx), "arrays")


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("base", "all"):
        main()
    if which in ("c1", "all"):
        main_c1()
    if which in ("edge", "all"):
        main_edge()
    if which in ("pbc", "all"):
        main_pbc()
    if which in ("dx", "all"):
        main_dx()
    if which in ("limits", "all"):
        main_limits()
