#!/usr/bin/env python3
"""Benchmark of the DDA solve hot path: time-to-residual 1e-5 per right-hand
side, FP64-checked, on the 128^3 sphere workload (m = 1.33+0.05i, x = 20,
QMRCCG, tol 1e-5).

A step solves one batch of R right-hand sides (orientations x 2 polarisations,
Euler angles uniform on SO(3) from a per-rank seed) until every RHS has an
FP64-recomputed true residual ||b - A x|| / ||b|| <= tol (RHS that pass the
FP32-MATVEC check but not the FP64 one are re-solved from their current x with
a tighter tolerance inside the step).  `value` is RHS per second with inputs
resident in HBM; `e2e` is the same metric through the C ABI with pinned host
buffers (H2D of b, x0, CXADIA and D2H of x inside the timed region).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference implementation of the path: the
reference CUDA library built unmodified from its sources (oracle/_ref), called
through its own C ABI one RHS at a time, on the same inputs.
"""
import argparse
import contextlib
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "ddscat-cuda_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "time-to-residual 1e-5 per RHS (FP64-checked), as RHS solved per second"
UNIT = "RHS/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--orient", type=int, default=64, help="orientations per rank (x2 polarisations = RHS per step)")
    ap.add_argument("--solver", default="qmrccg", choices=["qmrccg", "pbcgs2"])
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--maxit", type=int, default=4000)
    ap.add_argument("--policy", default="replace", choices=["replace", "restart"],
                    help="reliable-residual policy of the batched solve: residual replacement or restart")
    ap.add_argument("--qmr-form", default="symmetric", choices=["symmetric", "two-product"],
                    help="QMRCCG: one MATVEC per iteration (left Lanczos vectors = right ones, A^T = A) or the "
                         "reference's two-product form")
    ap.add_argument("--graph", default="on", choices=["on", "off"],
                    help="QMRCCG symmetric form with replacement: device-driven iterations launched as a CUDA graph")
    ap.add_argument("--ref-rhs", type=int, default=2,
                    help="RHS per step of the reference arm: a bounded sample of the batch, a different orientation's "
                         "pair of RHS each step (0: the whole batch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-q-check", action="store_true", help="skip the all-FP64 reference solve and Q errors")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or not f[0].isdigit() or int(f[0]) != self.idx:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


@contextlib.contextmanager
def quiet_stdout():
    """Silence C-level stdout (the reference library prints per-MATVEC lines)."""
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        yield
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg, local):
    if pg is None:
        return
    if pg.get_backend() == "nccl":
        pg.barrier(device_ids=[local])
    else:
        pg.barrier()


def max_over_ranks(pg, value):
    """Max of a per-rank scalar (the slowest rank's time) over the job."""
    if pg is None:
        return value
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def workload(args, rank):
    from ddscat_b200 import targets

    orients = targets.random_orientations(args.orient, seed=1000 + rank)
    prob = targets.make_problem(args.n, m=1.33 + 0.05j, x=20.0, orientations=orients)
    R = len(prob.incid)
    b = np.stack([prob.rhs(r) for r in range(R)])
    adia = np.stack([prob.adia(r) for r in range(R)])
    return prob, b, adia


def config(args, prob, R, world):
    return {"workload": f"{args.n}^3 sphere, m=1.33+0.05i, x=20, {args.solver.upper()} tol {args.tol:g}, "
                        f"{args.orient} orientations x 2 polarisations per rank",
            "n": args.n, "nat": prob.nat, "nat0": prob.nat0, "rhs_per_rank": R, "solver": args.solver,
            "polarisability": f"{prob.cmdpol} (isotropic material; CXAOFF = 0)",
            "tol": args.tol, "fp64_check": "GPU all-FP64 MATVEC true residual, every RHS, every step",
            "l2": "inputs larger than L2 (each RHS vector 3*NAT*8 B > 50 MB; working set > 1 GB)",
            "parallelism": f"replicas x{world} (independent RHS batches per GPU)",
            "reliable_residual_policy": getattr(args, "policy", "restart"),
            "qmr_form": getattr(args, "qmr_form", "two-product") if args.solver == "qmrccg" else None,
            "iteration_launch": ("CUDA graph, device-driven scalars" if getattr(args, "graph", "off") == "on"
                                 and args.solver == "qmrccg" else "host-driven")}


def algorithmic_bytes_per_matvec(prob, rhs_per_call):
    """8 B x [4*3*Mx*My*nz + 12*NAT0 + 6*(nx+1)(ny+1)(nz+1)/R] per RHS MATVEC:
    the half-padded spectrum round trip, x/y/CXADIA/CXAOFF, and the Green octant
    amortised over the RHS of one batched MATVEC."""
    nx, ny, nz = prob.nx, prob.ny, prob.nz
    return 8.0 * (12.0 * (2 * nx) * (2 * ny) * nz + 12.0 * prob.nat0 +
                  6.0 * (nx + 1) * (ny + 1) * (nz + 1) / max(rhs_per_call, 1.0))


def load_profile_traffic(n):
    """DRAM bytes per RHS-MATVEC from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", f"matvec_{n}cubed_ncu.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_rhs_matvec:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def cpu_model():
    """Host CPU model name (Linux /proc/cpuinfo), for the CPU baseline record."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(prob, ncompte_mean):
    """CPU restatement (the oracle, test infrastructure) timed on the host:
    a bounded sample of 3 MATVECs of the complex64 FFT operator at the full
    size (scipy.fft on all host threads, a random Green spectrum of the true
    shape), scaled by the GPU run's mean MATVEC count per RHS."""
    from oracle import ddscat_oracle as O

    nx, ny, nz = prob.nx, prob.ny, prob.nz
    rng = np.random.default_rng(0)
    shape = (6, 2 * nz, 2 * ny, 2 * nx)
    g = (rng.standard_normal(shape, dtype=np.float32) + 1j * rng.standard_normal(shape, dtype=np.float32))
    op = O.Operator(nx, ny, nz, g.astype(np.complex64), prob.iocc, dtype=np.complex64)
    occ = op.occ
    xc = O.gather_compact(prob.rhs(0), occ, prob.nat).astype(np.complex64)
    ac = O.gather_compact(prob.adia(0), occ, prob.nat).astype(np.complex64)
    oc = np.zeros_like(ac)
    op.apply_compact(xc, ac, oc)  # warm-up (plans, page faults)
    t0 = time.perf_counter()
    nmv = 3
    for _ in range(nmv):
        op.apply_compact(xc, ac, oc)
    t_mv = (time.perf_counter() - t0) / nmv
    per_rhs = t_mv * ncompte_mean
    return {"value": 1.0 / per_rhs, "unit": UNIT, "cores": os.cpu_count(), "cpu_model": cpu_model(), "kind": "port",
            "sample": f"{nmv} MATVECs of the complex64 oracle FFT operator at {nx}^3 (scipy.fft, "
                      f"{os.cpu_count()} threads), {t_mv:.3f} s each, scaled by {ncompte_mean:.1f} MATVECs per RHS",
            "c1_full_solve": cpu_c1_solve()}


def cpu_c1_solve():
    """A whole CPU solve timed end to end on the small sphere workload (32^3,
    m = 1.50+0.01i, x = 5, PBCGS2 at tol 1e-5, both polarisations): the
    oracle's complex64 FFT operator (scipy.fft, all host threads) inside the
    oracle's PBCGS2 recurrence (FP64 vectors and scalars)."""
    from ddscat_b200 import targets
    from oracle import ddscat_oracle as O

    prob = targets.make_problem(32, m=1.5 + 0.01j, x=5.0)
    k = prob.incid[0].k
    t0 = time.perf_counter()
    op = O.Operator.from_params(O.GreenParams(32, 32, 32, ak=tuple(float(np.float32(a)) for a in k)), prob.iocc,
                                dtype=np.complex64)
    t_green = time.perf_counter() - t0
    occ = op.occ
    zero = np.zeros(3 * op.nat0, dtype=np.complex64)
    its, times = [], []
    for r in range(len(prob.incid)):
        bc = O.gather_compact(prob.rhs(r), occ, prob.nat)
        ac = O.gather_compact(prob.adia(r), occ, prob.nat).astype(np.complex64)
        t0 = time.perf_counter()
        res = O.solve_pbcgs2(lambda v: op.apply_compact(v.astype(np.complex64), ac, zero).astype(np.complex128),
                             bc, np.zeros_like(bc), 500, 1e-5)
        times.append(time.perf_counter() - t0)
        its.append(res.itno)
    return {"workload": "32^3 sphere, m=1.50+0.01i, x=5, PBCGS2 tol 1e-5, 1 orientation x 2 polarisations",
            "s_per_rhs": float(np.mean(times)), "rhs_per_s": 1.0 / float(np.mean(times)),
            "iterations": its, "green_build_s": t_green, "threads": os.cpu_count(), "cpu_model": cpu_model()}


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import torch

    import ddscat_b200 as D

    world, rank, local, pg = dist_init()
    prob, b, adia = workload(args, rank)
    R = b.shape[0]
    dda = D.DDA("fft3d")
    dda.prepare_green(prob.nx, prob.ny, prob.nz, prob.iocc, prob.incid[0].k)
    dev = torch.device("cuda", local)
    bd = torch.from_numpy(b).to(dev)
    ad = torch.from_numpy(adia).to(dev)
    xd = torch.zeros_like(bd)
    stats = {"iters": [], "ncompte": [], "res64": [], "resolves": 0, "mv_ms": 0.0, "mv_rhs": 0, "mv_calls": 0}

    def solve_to_fp64(bx, xx, ax, on_device, on_solved=None):
        """One step: batched solve, FP64 true residuals, re-solve failures.
        on_solved() runs once the first solve has returned (its x is final
        unless an RHS fails the FP64 check); returns (out, res, re-solve rounds)."""
        rep = args.policy == "replace"
        sym = args.solver == "qmrccg" and args.qmr_form == "symmetric"
        gr = sym and rep and args.graph == "on"
        out = dda.solve_batch(args.solver, bx, xx, ax, None, maxit=args.maxit, tol=args.tol, replace=rep,
                              symmetric=sym, graph=gr)
        if on_solved is not None:
            on_solved()
        ms, rhs, calls = dda.last_solve_stats()
        stats["mv_ms"] += ms
        stats["mv_rhs"] += rhs
        stats["mv_calls"] += calls
        res = dda.residual_f64(bx, xx, ax)
        tol = args.tol
        rounds = 0
        while np.any(res > args.tol) and rounds < 4:
            bad = np.flatnonzero(res > args.tol)
            tol *= 0.5
            sub = (lambda a: a[bad].contiguous()) if on_device else (lambda a: np.ascontiguousarray(a[bad]))
            xs = sub(xx)
            o2 = dda.solve_batch(args.solver, sub(bx), xs, sub(ax), None, maxit=args.maxit, tol=tol, replace=rep,
                                 symmetric=sym, graph=gr)
            xx[bad] = xs
            out.itno[bad] += o2.itno
            out.ncompte[bad] += o2.ncompte
            res[bad] = dda.residual_f64(sub(bx), xs, sub(ax))
            stats["resolves"] += len(bad)
            rounds += 1
        return out, res, rounds

    def step_dev(record):
        xd.zero_()
        out, res, _ = solve_to_fp64(bd, xd, ad, True)
        if record:
            stats["iters"] += list(out.itno)
            stats["ncompte"] += list(out.ncompte)
            stats["res64"] += list(res)
        return out

    for _ in range(args.warmup):
        step_dev(False)
    stats.update(mv_ms=0.0, mv_rhs=0, mv_calls=0)
    clocks = ClockSampler(local)
    barrier(pg, local)
    torch.cuda.synchronize()
    clocks.start()
    l0 = dda.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step_dev(True)
    e1.record()
    torch.cuda.synchronize()
    barrier(pg, local)
    launches = dda.launch_count() - l0
    clk = clocks.stop()
    elapsed = max_over_ranks(pg, e0.elapsed_time(e1) / 1000.0)
    total_rhs = R * args.steps * world
    value = total_rhs / elapsed
    mv_stats = (stats["mv_ms"], stats["mv_rhs"], stats["mv_calls"])

    # end-to-end through the C ABI: every step copies b, x0 and CXADIA from
    # pinned host memory to the device, solves and FP64-checks on those copies
    # (device-pointer calls of the batched API, same stream) and reads the
    # solutions back to pinned host memory
    bh = torch.from_numpy(b).pin_memory()
    ah = torch.from_numpy(adia).pin_memory()
    xh = torch.zeros_like(bh).pin_memory()
    xo = torch.empty_like(bh).pin_memory()
    be, ae, xe = torch.empty_like(bd), torch.empty_like(ad), torch.empty_like(bd)

    # the read-back of x runs on a side stream, overlapped with the FP64
    # residual check of the same x (both only read it); it is repeated if a
    # re-solve changed x, and every step waits for it
    d2h = torch.cuda.Stream(device=dev)

    def start_d2h():
        ev = torch.cuda.Event()
        ev.record()
        d2h.wait_event(ev)
        with torch.cuda.stream(d2h):
            xo.copy_(xe, non_blocking=True)

    def step_host():
        be.copy_(bh, non_blocking=True)
        ae.copy_(ah, non_blocking=True)
        xe.copy_(xh, non_blocking=True)
        _, _, rounds = solve_to_fp64(be, xe, ae, True, start_d2h)
        torch.cuda.current_stream().wait_stream(d2h)
        if rounds:
            xo.copy_(xe)

    step_host()  # warm-up of the host path
    # the end-to-end figure over at most 5 steps of the same batch (each step is
    # a whole 128-RHS solve with its copies; this bounds the run time)
    e2e_steps = min(args.steps, 5)
    barrier(pg, local)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(e2e_steps):
        step_host()
    f1.record()
    torch.cuda.synchronize()
    barrier(pg, local)
    e2e_elapsed = max_over_ranks(pg, f0.elapsed_time(f1) / 1000.0)
    vec = 3 * prob.nat * 8
    h2d = R * vec * 3  # b, x0 and CXADIA
    d2h = R * vec      # x
    del bh, ah, xh, xo, be, ae, xe  # host-path buffers: free for the checks below
    torch.cuda.empty_cache()

    # The drop-in path as unchanged DDSCAT calls it: this library's own
    # ddscat_cuda_solve_<solver>_f32 (the reference's entry point, its
    # recurrence and restart rule) with host buffers, one RHS per call, on the
    # same bounded sample as the reference arm (--ref-rhs RHS per step, a
    # different orientation each step); console lines off, as in benchmarks.
    abi = None
    if rank == 0 and world == 1:
        nref = R if args.ref_rhs <= 0 else min(args.ref_rhs, R)
        aoff0 = np.zeros(b.shape[1], dtype=np.complex64)
        dda.lib.ddscat_b200_set_verbose(0)
        dda.solve(args.solver, b[0], adia[0], aoff0, maxit=args.maxit, tol=args.tol)  # warm-up
        its, ncs = [], []
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for st in range(args.steps):
            for j in range(nref):
                r = (nref * st + j) % R
                o = dda.solve(args.solver, b[r], adia[r], aoff0, maxit=args.maxit, tol=args.tol)
                its.append(o.itno)
                ncs.append(o.ncompte)
        g1.record()
        torch.cuda.synchronize()
        dda.lib.ddscat_b200_set_verbose(-1)
        abi_s = g0.elapsed_time(g1) / 1000.0
        abi = {"value": nref * args.steps / abi_s, "unit": UNIT,
               "entry_point": f"ddscat_cuda_solve_{args.solver}_f32 (the reference's C ABI, host buffers, one RHS per call)",
               "rhs_per_step": nref, "steps": args.steps, "iterations_mean": float(np.mean(its)),
               "matvecs_per_rhs_mean": float(np.mean(ncs)),
               "sample": "the reference arm's sample: step s solves RHS nref*s .. nref*s+nref-1 (mod the batch)"}

    # Q errors of the FP32 solutions against the same batch solved all-FP64 on
    # the GPU (outside the timed regions; every rank checks its own batch)
    qerr = None
    if not args.no_q_check:
        nat = prob.nat
        occ = prob.occ

        def compact(v):
            return np.concatenate([v[c * nat:(c + 1) * nat][occ] for c in range(3)])

        x32 = xd.cpu().numpy()
        x64 = np.zeros(b.shape, dtype=np.complex128)
        its64 = []
        # FP64 solves in chunks of 16 RHS (complex-double Krylov vectors of the
        # whole 128-RHS batch do not fit beside the FP32 batch's buffers)
        for c0 in range(0, R, 16):
            c1 = min(R, c0 + 16)
            xc = np.zeros((c1 - c0, b.shape[1]), dtype=np.complex128)
            o64 = dda.solve_batch_f64(args.solver, np.ascontiguousarray(b[c0:c1]), xc, np.ascontiguousarray(adia[c0:c1]),
                                      None, maxit=args.maxit, tol=1e-8, replace=args.policy == "replace",
                                      symmetric=args.solver == "qmrccg" and args.qmr_form == "symmetric")
            x64[c0:c1] = xc
            its64 += list(o64.itno)
        worst = {"cabs": 0.0, "cext": 0.0, "cpha": 0.0}
        zero = np.zeros(3 * prob.nat0, dtype=np.complex64)
        for r in range(R):
            k = prob.incid[r].k
            ec, ac = compact(b[r]), compact(adia[r])
            q32 = dda.evalq(k, use_resident=0, e=ec, p=compact(x32[r]), adia=ac, aoff=zero)
            q64 = dda.evalq(k, use_resident=0, e=ec, p=compact(x64[r]).astype(np.complex64), adia=ac, aoff=zero)
            for key, a, c in zip(("cabs", "cext", "cpha"), q32, q64):
                worst[key] = max(worst[key], abs(a - c) / max(abs(c), 1e-300))
        # S_ij on 0..180 deg at 1 deg in two scattering planes per orientation:
        # FP32 (SCAT amplitudes of the FP32 solutions) against FP64 (FP64
        # amplitudes of the FP64 solutions), both through the Mueller entry points
        from ddscat_b200 import targets as T
        s11_err, sij_err, sij_glob, ndir = 0.0, 0.0, 0.0, 0
        csca_err, g_err, navg = 0.0, 0.0, 0
        for o in range(R // 2):
            r0, r1 = 2 * o, 2 * o + 1
            k = prob.incid[r0].k
            aks, em1, em2 = T.scattering_planes(k, prob.incid[r0].e)
            ndir = aks.shape[0]
            f32 = []
            for r in (r0, r1):
                dda.evalq(k, use_resident=0, e=compact(b[r]), p=compact(x32[r]), adia=compact(adia[r]), aoff=zero)
                sc = dda.scat(k, prob.incid[r].e, prob.x0, etasca=0.5, aks=aks.astype(np.float32),
                              em1=em1.astype(np.float32), em2=em2.astype(np.float32))
                f32.append((sc["f1"], sc["f2"]))
                # Qsca and g of the FP32 solution (FP32 phases, FP64 sums) against the
                # FP64 solution's (FP64 phases and sums), same directions and weights
                s64 = dda.scat_csca_f64(np.ascontiguousarray(x64[r:r + 1]), k, prob.incid[r].e, prob.x0, etasca=0.5)
                c64 = float(s64["csca"][0])
                csca_err = max(csca_err, abs(sc["csca"] - c64) / c64)
                g_err = max(g_err, abs(sc["cscag"][0] / sc["csca"] - float(s64["cscag"][0, 0]) / c64))
                navg = int(s64["navg"][0])
            _, m32 = dda.mueller(k, prob.incid[r0].e, prob.incid[r1].e, em2.astype(np.float32),
                                 f32[0][0], f32[0][1], f32[1][0], f32[1][1])
            g1, g2 = dda.scat_amplitudes_f64(np.ascontiguousarray(x64[r0:r1 + 1]), k, aks, em1, em2, prob.x0)
            _, m64 = dda.mueller_f64(k, prob.incid[r0].e, prob.incid[r1].e, em2, g1[0], g2[0], g1[1], g2[1])
            s11 = m64[:, 0, 0]
            s11_err = max(s11_err, float(np.max(np.abs(m32[:, 0, 0] - s11) / s11)))
            sij_err = max(sij_err, float(np.max(np.abs(m32 - m64) / s11[:, None, None])))
            sij_glob = max(sij_glob, float(np.max(np.abs(m32 - m64)) / np.max(s11)))
        qerr = {"cabs_max_rel": worst["cabs"], "cext_max_rel": worst["cext"], "cpha_max_rel": worst["cpha"],
                "csca_max_rel": csca_err, "g_max_abs": g_err,
                "csca_g_quadrature": f"SCAT integration at ETASCA 0.5, NAVG {navg} directions",
                "s11_max_rel": s11_err, "sij_max_abs_over_s11": sij_err, "sij_max_abs_over_max_s11": sij_glob,
                "s_ij_directions": f"theta 0..180 deg at 1 deg in 2 planes ({ndir}) x {R // 2} orientations",
                "rhs": R, "fp64_solve": f"{args.solver.upper()} all-FP64 on the GPU, tol 1e-8, FP64 far-field sums",
                "fp64_iterations_mean": float(np.mean(its64))}

    if rank == 0:
        ncm = float(np.mean(stats["ncompte"]))
        rhs_per_call = mv_stats[1] / max(mv_stats[2], 1)
        alg = algorithmic_bytes_per_matvec(prob, rhs_per_call)
        ms_per_rhs_mv = mv_stats[0] / max(mv_stats[1], 1)
        achieved = alg / (ms_per_rhs_mv * 1e-3) / 1e9
        peak, peak_kind = measured_peak()
        traffic = load_profile_traffic(args.n)
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(prob, ncm)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed * 1000.0 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP32 complex bulk, FP64 dots and checks)",
            "data": "synthetic (seeded sphere target and incident fields)", "config": config(args, prob, R, world),
            "ms_per_rhs": elapsed * 1000.0 / (R * args.steps),
            "iterations_mean": float(np.mean(stats["iters"])), "matvecs_per_rhs_mean": ncm,
            "fp64_residual_max": float(np.max(stats["res64"])), "fp64_resolved_rhs": stats["resolves"],
            "roofline": {"bound": "hbm", "kernel": "MATVEC (5 register-FFT passes, all RHS of one batched call)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": None if traffic is None else traffic,
                         # measured DRAM bytes (ncu, per RHS-MATVEC) over the event-timed MATVEC
                         "traffic_gbs": None if traffic is None else traffic / (ms_per_rhs_mv * 1e-3) / 1e9,
                         "traffic_frac": None if traffic is None else traffic / (ms_per_rhs_mv * 1e-3) / 1e9 / peak,
                         "algorithmic_bytes_per_rhs_matvec": alg, "ms_per_rhs_matvec": ms_per_rhs_mv,
                         "rhs_per_matvec_call": rhs_per_call},
            "cpu_baseline": cpu,
            "e2e": {"value": R * e2e_steps * world / e2e_elapsed, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "gpu_launches": launches, "clocks": clk, "abi_single_rhs": abi,
            "q_error_vs_fp64": qerr,
        }
        print(json.dumps(line), flush=True)
    dda.release()
    if pg is not None:
        pg.destroy_process_group()


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    import ctypes as ct

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    path = os.path.join(ROOT, "oracle", "_ref", "libddscat_ref_fft3d.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference", "unavailable": f"reference library not built ({path})"}))
        return
    lib = ct.CDLL(path, mode=ct.RTLD_LOCAL)
    P = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
    lib.ddscat_cuda_prepare_green_f32.argtypes = [ct.c_int] * 7 + [ct.c_float] * 9 + [ct.c_void_p]
    fn = getattr(lib, f"ddscat_cuda_solve_{args.solver}_f32")
    fn.argtypes = [ct.c_void_p] * 4 + [ct.c_int, ct.c_int, ct.c_float] + [ct.c_void_p] * 3
    prob, b, adia = workload(args, 0)
    aoff = np.zeros(b.shape[1], dtype=np.complex64)
    nref = b.shape[0] if args.ref_rhs <= 0 else min(args.ref_rhs, b.shape[0])
    k = prob.incid[0].k
    with quiet_stdout():
        rc = lib.ddscat_cuda_prepare_green_f32(prob.nx, prob.ny, prob.nz, 0, prob.nat, prob.nat0, 0, 0.0, 0.0, 0.0,
                                               float(k[0]), float(k[1]), float(k[2]), 1.0, 1.0, 1.0, P(prob.iocc))
    if rc != 0:
        print(json.dumps({"impl": "reference", "unavailable": f"reference prepare_green failed with status {rc}"}))
        return
    iters = []
    R = b.shape[0]
    nstep = [0]

    def step(record, count=nref):
        # a different orientation's RHS each step, so the sample spreads over the batch
        first = nref * nstep[0]
        nstep[0] += 1
        for j in range(count):
            r = (first + j) % R
            x = np.zeros(b.shape[1], dtype=np.complex64)
            it, tole, nc = ct.c_int(), ct.c_float(), ct.c_int()
            rr = fn(P(b[r]), P(x), P(adia[r]), P(aoff), b.shape[1], args.maxit, args.tol, ct.byref(it),
                    ct.byref(tole), ct.byref(nc))
            if rr != 0:
                raise RuntimeError(f"reference solve failed with status {rr}")
            if record:
                iters.append(it.value)

    with quiet_stdout():
        for _ in range(args.warmup):
            step(False, 1)  # warm-up: one RHS per step
        nstep[0] = 0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step(True)
        e1.record()
        torch.cuda.synchronize()
    elapsed = e0.elapsed_time(e1) / 1000.0
    value = nref * args.steps / elapsed
    sample = (f"reference ddscat_matvec_cuda.cu built unmodified (oracle/Makefile), {args.solver.upper()} through its "
              f"own C ABI with host buffers, one RHS at a time, {nref} RHS per step (step s solves RHS "
              f"{nref}s..{nref}s+{nref - 1} mod {R} of the workload's batch), its own restart policy; the reference "
              f"implementation of this path runs on the GPU, its host side on 1 thread")
    cfg = config(args, prob, R, world)
    cfg["reference_rhs_per_step"] = nref
    cfg["reliable_residual_policy"] = "restart (the reference's own)"
    cfg["qmr_form"] = "two-product (the reference's own)" if args.solver == "qmrccg" else None
    cfg["fp64_check"] = "none: the reference returns its own FP32 residual TOLE (true residual at its reliable checks)"
    cfg["iteration_launch"] = ("host-driven, one RHS per call, a host round trip per inner-product group "
                               "(the reference's own)")
    vec = b.shape[1] * 8
    h2d = nref * 4 * vec  # b, x0, CXADIA and CXAOFF copied in by every solve call
    d2h = nref * vec      # x copied out
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed * 1000.0 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 (FP32 complex bulk, FP64 dots)",
            "data": "synthetic (seeded sphere target and incident fields)", "config": cfg, "impl": "reference",
            "iterations_mean": float(np.mean(iters)),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "cpu_model": cpu_model(), "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "copies": "inside the reference's solve call (host buffers in, solution out), every step"}}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
