"""Many targets of uneven size solved together (ddscat_b200_multi_solve_f32):
the C4 configuration, 40 seeded random ellipsoids with lattice sides drawn
uniformly from 24 to 96 per axis, semi-axes filling 0.6-1.0 of the box,
Re m ~ U[1.2, 1.8], Im m ~ U[0.001, 0.1], x = 0.15 * (largest side), two
polarisations each (80 RHS), PBCGS2.  Each target is solved on its drawn
lattice sides (even sides run on padded register-FFT lengths, odd ones on
the generic z-first pipeline).  Every RHS converges; for three targets the
FP64 true residual is <= 1.2*TOL, the solutions match the single-target
batched solve to 20*TOL, and Cext, Cabs (EVALQ) and Csca (SCAT) of the FP32
solutions are within 1e-4 of those of the all-FP64 batched solve."""
import numpy as np
import pytest

import ddscat_b200 as D
from ddscat_b200 import targets

TOL = 1e-5


def c4_targets(count=40, seed=0, grid="exact"):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        sides = [int(v) for v in rng.integers(24, 97, size=3)]
        fill = rng.uniform(0.6, 1.0, size=3)
        semi = tuple(fill[a] * sides[a] / 2.0 for a in range(3))
        m = complex(rng.uniform(1.2, 1.8), rng.uniform(0.001, 0.1))
        x = 0.15 * max(sides)
        dims, iocc = targets.embed_ellipsoid(sides, semi, grid)
        out.append(targets.make_problem(*dims, m=m, x=x, iocc=iocc))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("graph", [False, True])
def test_c4_uneven_multi_target(graph):
    """graph=True: the PBCGS2 iterations of all targets run device-driven as
    branches of one captured graph, launched once per Krylov step."""
    probs = c4_targets()
    items = []
    for p in probs:
        b = np.stack([p.rhs(r) for r in range(2)])
        items.append({"dims": (p.nx, p.ny, p.nz), "iocc": p.iocc, "ak": p.incid[0].k, "b": b,
                      "x": np.zeros_like(b), "adia": np.stack([p.adia(r) for r in range(2)])})
    dda = D.DDA()
    out = dda.multi_solve(items, "pbcgs2", maxit=3000, tol=TOL, symmetric=False, graph=graph)
    assert out.itno.size == 80 and np.all(out.status == 0) and np.all(out.tole <= TOL)
    sizes = [p.nat for p in probs]
    for t in (int(np.argmin(sizes)), int(np.argsort(sizes)[len(sizes) // 2]), int(np.argmax(sizes))):
        p, it = probs[t], items[t]
        dda.prepare_green(p.nx, p.ny, p.nz, p.iocc, p.incid[0].k)
        r64 = dda.residual_f64(it["b"], it["x"], it["adia"])
        assert np.all(r64 <= 1.2 * TOL), (t, r64)
        xs = np.zeros_like(it["b"])
        dda.solve_batch("pbcgs2", it["b"], xs, it["adia"], maxit=3000, tol=TOL, replace=True)
        for r in range(2):
            assert np.linalg.norm(xs[r] - it["x"][r]) / np.linalg.norm(xs[r]) < 20 * TOL
        # Q values of the FP32 solutions against the all-FP64 batched solve
        x64 = np.zeros(it["b"].shape, dtype=np.complex128)
        o64 = dda.solve_batch_f64("pbcgs2", it["b"], x64, it["adia"], maxit=4000, tol=1e-9, replace=True)
        assert np.all(o64.status == 0)
        nat, occ = p.nat, p.occ
        comp = lambda v: np.concatenate([v[c * nat:(c + 1) * nat][occ] for c in range(3)])  # noqa: E731
        zero = np.zeros(3 * p.nat0, dtype=np.complex64)
        k = p.incid[0].k
        for r in range(2):
            e, a = comp(it["b"][r]), comp(it["adia"][r])
            q32 = dda.evalq(k, use_resident=0, e=e, p=comp(it["x"][r]), adia=a, aoff=zero)
            sc32 = dda.scat(k, p.incid[r].e, p.x0, etasca=0.5)
            q64 = dda.evalq(k, use_resident=0, e=e, p=comp(x64[r]).astype(np.complex64), adia=a, aoff=zero)
            s64 = dda.scat_csca_f64(np.ascontiguousarray(x64[r:r + 1]), k, p.incid[r].e, p.x0, etasca=0.5)
            for g, w in zip(q32[:2], q64[:2]):
                assert abs(g - w) <= 1e-4 * abs(w), (t, r, g, w)
            assert abs(sc32["csca"] - s64["csca"][0]) <= 1e-4 * s64["csca"][0], (t, r)
    dda.release()


@pytest.mark.gpu
def test_multi_target_graph_solves_concurrent_equal_serial():
    """The graph-driven QMRCCG of several targets run by concurrent host threads
    (one CUDA stream each) gives the same iterations and solutions as the same
    solves run one after another: every target's state reaches the GPU in its
    own stream order."""
    probs = c4_targets(count=8, seed=3)

    def items():
        out = []
        for p in probs:
            b = np.stack([p.rhs(r) for r in range(2)])
            out.append({"dims": (p.nx, p.ny, p.nz), "iocc": p.iocc, "ak": p.incid[0].k, "b": b,
                        "x": np.zeros_like(b), "adia": np.stack([p.adia(r) for r in range(2)])})
        return out

    dda = D.DDA()
    one, eight = items(), items()
    a = dda.multi_solve(one, "qmrccg", maxit=3000, tol=TOL, symmetric=True, graph=True, nthreads=1, check=False)
    b = dda.multi_solve(eight, "qmrccg", maxit=3000, tol=TOL, symmetric=True, graph=True, nthreads=8, check=False)
    assert np.all(a.status == 0) and np.all(b.status == 0)
    np.testing.assert_array_equal(a.itno, b.itno)
    for u, v in zip(one, eight):
        np.testing.assert_array_equal(u["x"], v["x"])
    dda.release()


@pytest.mark.gpu
def test_multi_wavelength_one_target():
    """Many wavelengths of one target in one call: each wavelength has its own
    Green tensor, so it enters as a target of its own (same lattice and
    occupancy, wave number x / a_eff); 3 wavelengths x 2 orientations x 2
    polarisations, PBCGS2 as graph branches.  Every RHS converges and matches
    the single-target batched solve of its wavelength to 20*TOL."""
    base = targets.make_problem(24, 20, 16, m=1.5 + 0.02j, x=2.0)
    probs = [targets.make_problem(24, 20, 16, m=1.5 + 0.02j, x=x, iocc=base.iocc,
                                  orientations=targets.random_orientations(2, seed=7)) for x in (2.0, 3.5, 5.0)]
    items = []
    for p in probs:
        b = np.stack([p.rhs(r) for r in range(4)])
        items.append({"dims": (p.nx, p.ny, p.nz), "iocc": p.iocc, "ak": p.incid[0].k, "b": b,
                      "x": np.zeros_like(b), "adia": np.stack([p.adia(r) for r in range(4)])})
    # the orientations rotate k: every RHS of a target must share |k| (one Green tensor per target)
    for p in probs:
        assert np.allclose([np.linalg.norm(i.k) for i in p.incid], np.linalg.norm(p.incid[0].k))
    dda = D.DDA()
    out = dda.multi_solve(items, "pbcgs2", maxit=2000, tol=TOL, symmetric=False, graph=True)
    assert out.itno.size == 12 and np.all(out.status == 0) and np.all(out.tole <= TOL)
    for p, it in zip(probs, items):
        dda.prepare_green(p.nx, p.ny, p.nz, p.iocc, p.incid[0].k)
        xs = np.zeros_like(it["b"])
        dda.solve_batch("pbcgs2", it["b"], xs, it["adia"], maxit=2000, tol=TOL, replace=True)
        for r in range(4):
            assert np.linalg.norm(xs[r] - it["x"][r]) / np.linalg.norm(xs[r]) < 20 * TOL
    dda.release()
