"""MATVEC timing of a prepared sphere target (command-line utility).

  python -m ddscat_b200.timing [--n 128] [--nrhs 1] [--iters 10] [--layout fft3d|slices]
                               [--cwhat N|C] [--x 20]

Prepares an n^3 sphere (m = 1.33+0.05i, size parameter x, Green tensor built
on the GPU), then times `iters` device-resident MATVECs of `nrhs` right-hand
sides each through ddscat_b200_matvec_timing (3 untimed warm-up calls, CUDA
events on the library stream) and prints one JSON line with the mean time per
call and per RHS.  Small enough to run under a kernel profiler: the MATVEC
kernels of one call are launched once per call, in pass order.
"""
from __future__ import annotations

import argparse
import json

from . import DDA
from . import targets


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--nrhs", type=int, default=1)
    ap.add_argument("--iters", type=int, default=10)
    ap.add_argument("--layout", default="fft3d", choices=["fft3d", "slices"])
    ap.add_argument("--cwhat", default="N", choices=["N", "C"])
    ap.add_argument("--x", type=float, default=20.0)
    a = ap.parse_args(argv)
    prob = targets.make_problem(a.n, m=1.33 + 0.05j, x=a.x)
    dda = DDA(a.layout)
    dda.prepare_green(a.n, a.n, a.n, prob.iocc, prob.incid[0].k)
    ms = dda.matvec_ms(a.nrhs, a.iters, a.cwhat)
    print(json.dumps({"n": a.n, "nat": prob.nat, "nat0": prob.nat0, "layout": a.layout, "nrhs": a.nrhs,
                      "iters": a.iters, "ms_per_call": ms, "ms_per_rhs": ms / a.nrhs}), flush=True)
    dda.release()


if __name__ == "__main__":
    main()
