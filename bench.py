#!/usr/bin/env python
"""Benchmark: solves/s of GeMSLR-preconditioned FGMRES on one B200 per rank.

Workload (the headline configuration): 3D 7-point Laplacian on a 128^3 grid
(2,097,152 unknowns, 14.6M nonzeros, the reference's stencil), b = A x_true
with x_true = 2u - 1 seeded; 4 GeMSLR levels, ILUT drop 1e-3 / 200 per row,
rank 16 per level, inner Schur FGMRES on level 0 (tol 1e-2, 5 steps),
FGMRES(50) to relative residual 1e-8 from x0 = 0.

Setup (untimed).  By default the preconditioner is the reference's own:
GemslrClass::Setup of the reference, compiled from its sources into
oracle/_ref, runs once on all host threads, writes its post-setup structures,
and they are imported through the C ABI (pgx_gemslr_set_*) exactly as a
reference-side driver would hand them over.  The same run solves the first
right-hand side on the CPU, which gives the reference's solution x_ref, its
iteration count and the CPU baseline's time.  ``--setup own`` uses this
library's host setup (pgx_gemslr_setup) instead.

A "step" is one batch of --batch right-hand sides (b_r = A x_r, x_r seeded),
each solved completely from x0 = 0, concurrently over the one resident
preconditioner (pgx_gemslr_solve_batch): slot 0 takes one, every further slot
--lanes of them in lockstep (their triangular passes merged); value =
solves/s.

  python bench.py [--gpus N --steps K --warmup W] [--precision mixed|fp64] [--setup reference|own]
  python bench.py --impl reference ...   (the reference CPU solver, oracle/_ref, full solves)
  python bench.py --impl reference --ref-mode throughput   (one single-threaded reference per host thread)

Under torchrun (N > 1) every rank solves its own replica on its own GPU; the
solve does not shard, so there is no collective in the data path; the
device time is reduced with MAX over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pargemslr_b200 import params as P  # noqa: E402
from pargemslr_b200 import pgxd, problems  # noqa: E402
from pargemslr_b200._abi import LOCATION_DEVICE, LOCATION_HOST  # noqa: E402

GRID = (128, 128, 128)
WORKLOAD = "lap3d_128"
SEED = 7


def metric_name() -> str:
    return "solves/s (GeMSLR-FGMRES(50), rel-res 1e-8, 3D Laplacian %d^3)" % GRID[0]


def workload_config(setup: str) -> dict:
    """The `config` both arms print: the same workload, so their lines compare like for like."""
    n = GRID[0] * GRID[1] * GRID[2]
    who = {"reference": "the reference's GemslrClass::Setup (oracle/_ref) on all host threads, untimed",
           "parallel": "the reference's ParallelGemslrClass::Setup at one rank (oracle/_ref/pgx_ref_driver_par), its "
                       "per-level permutations composed, untimed"}.get(
        setup, "this library's host setup (pgx_gemslr_setup), untimed")
    return {"workload": "3D 7-point Laplacian %d^3 (n=%d), 4 levels, ILUT 1e-3/200, rank 16, inner Schur FGMRES(5) "
                        "tol 1e-2, FGMRES(50) to rel-res 1e-8 from x0 = 0, b = A x_true (x_true = 2u-1, seeded)"
                        % (GRID[0], n),
            "setup": who}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="pgx_clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.out.name) as f:
            for line in f:
                parts = [t.strip() for t in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.out.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(lanes: int):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary (None if not captured)."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None
    return d.get("lanes%d" % lanes)


def max_over_ranks(value: float, device) -> float:
    """The largest value over all ranks (a one-element all-reduce; identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def log(msg: str) -> None:
    """Progress of the phases on stderr (the JSON line alone goes to stdout)."""
    print("[bench %.1fs] %s" % (time.time() - _T0, msg), file=sys.stderr, flush=True)


_T0 = time.time()


def build_problem():
    A = problems.laplacian(*GRID)
    n = A[0].size - 1
    xt = problems.x_true(n, SEED)
    b = problems.spmv(A, xt)
    return A, n, b, xt


# ------------------------------------------------------------ reference leg
def _ref_driver() -> str:
    return os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver")


def _ref_command(out: str, xtrue_path: str, n_threads: int, solves: int, dump: bool):
    p = P.workload_params(WORKLOAD)
    cmd = [_ref_driver(), "--out", out, "--lap", *[str(g) for g in GRID], "0", "0", "0", "0", "--xtrue", xtrue_path,
           "--threads", str(n_threads), "--solve", "--repeat", str(solves)]
    if dump:
        cmd.append("--dump")
    for i, v in enumerate(p):
        cmd += ["--param", f"{i}={float(v)!r}"]
    env = dict(os.environ, OMP_NUM_THREADS=str(n_threads), OPENBLAS_NUM_THREADS="1")
    return cmd, env


def _ref_result(out: str, wall: float):
    res = {}
    with open(os.path.join(out, "result.txt")) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            res[k] = v
    times = [float(t) for t in res["solve_times"].split(",")]
    return {"dir": out, "times": times, "iters": int(res["iters"]), "setup_s": float(res["setup_s"]),
            "true_rel_res": float(res["true_rel_res"]), "wall_s": wall}


def _ref_inputs():
    if not os.path.exists(_ref_driver()):
        return None
    d = tempfile.mkdtemp(prefix="pgx_ref_")
    n = GRID[0] * GRID[1] * GRID[2]
    path = os.path.join(d, "xtrue.bin")
    pgxd.write(path, {"x_true": problems.x_true(n, SEED)})
    return d, path


def reference_run(n_threads: int, solves: int, dump: bool):
    """The reference CPU solver (oracle/_ref) on the workload: its setup on n_threads threads, then `solves` full
    FGMRES solves of b = A x_true (x_true seeded as the first right-hand side of the GPU arm), each from x0 = 0.
    With dump, its post-setup structures are written for import (setup.bin), with b (problem.bin) and the solution
    (solution.bin).  Returns (result, None) or (None, why)."""
    inp = _ref_inputs()
    if inp is None:
        return None, "oracle/_ref/pgx_ref_driver not built"
    out, xtrue_path = inp
    cmd, env = _ref_command(out, xtrue_path, n_threads, solves, dump)
    t0 = time.time()
    subprocess.run(cmd, check=True, env=env, stdout=subprocess.DEVNULL)
    return _ref_result(out, time.time() - t0), None


def reference_run_parallel_class(n_threads: int):
    """The reference's ParallelGemslrClass at one rank (oracle/_ref/pgx_ref_driver_par) on the workload with the
    GeMSLR global preconditioner: its setup (exported with each level's transfer permutation, setup_par.bin), one
    FGMRES solve of b = A x_true from x0 = 0, b and the solution.  Returns (result, None) or (None, why)."""
    drv = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver_par")
    if not os.path.exists(drv):
        return None, "oracle/_ref/pgx_ref_driver_par not built"
    d = tempfile.mkdtemp(prefix="pgx_refpar_")
    n = GRID[0] * GRID[1] * GRID[2]
    xf = os.path.join(d, "xtrue.bin")
    pgxd.write(xf, {"x_true": problems.x_true(n, SEED)})
    p = P.workload_params(WORKLOAD)
    p[P.PRECOND_GLOBAL_PRECOND] = 2  # GeMSLR (the parallel drivers' GEMSLR option)
    cmd = [drv, "--out", d, "--lap", *[str(g) for g in GRID], "0", "0", "0", "0", "--xtrue", xf, "--threads",
           str(n_threads), "--dump", "--solve"]
    for i, v in enumerate(p):
        cmd += ["--param", f"{i}={float(v)!r}"]
    t0 = time.time()
    subprocess.run(cmd, check=True, env=dict(os.environ, OMP_NUM_THREADS=str(n_threads), OPENBLAS_NUM_THREADS="1"),
                   stdout=subprocess.DEVNULL)
    res = {}
    with open(os.path.join(d, "result.txt")) as f:
        for line in f:
            k, v = line.strip().split("=", 1)
            res[k] = v
    return {"dir": d, "times": [float(res["solve_s"])], "iters": int(res["iters"]), "setup_s": float(res["setup_s"]),
            "true_rel_res": float(res["true_rel_res"]), "wall_s": time.time() - t0, "parallel": True}, None


def reference_runs_parallel(procs: int, solves: int):
    """Throughput form of the reference baseline: `procs` single-threaded reference processes at once, each
    setting up and solving the same workload on its own, as independent solves on the host's cores would run.
    Returns one result per process."""
    inp = _ref_inputs()
    if inp is None:
        return None, "oracle/_ref/pgx_ref_driver not built"
    d, xtrue_path = inp
    runs = []
    t0 = time.time()
    for k in range(procs):
        out = os.path.join(d, f"p{k}")
        os.makedirs(out)
        cmd, env = _ref_command(out, xtrue_path, 1, solves, False)
        runs.append((out, subprocess.Popen(cmd, env=env, stdout=subprocess.DEVNULL)))
    codes = [proc.wait() for _, proc in runs]
    wall = time.time() - t0
    if any(codes):
        return None, f"reference processes exited with {codes}"
    return [_ref_result(out, wall) for out, _ in runs], None


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    solves = args.warmup + args.steps
    if args.ref_mode == "throughput":
        rs, why = reference_runs_parallel(threads, solves)
        if rs is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        # each process's solves/s over its timed solves, summed over the processes running at once
        value = sum(1.0 / statistics.mean(r["times"][args.warmup:]) for r in rs)
        t_solve = 1.0 / value
        r = rs[0]
        timed_s = max(sum(x["times"][args.warmup:]) for x in rs)
        sample = (f"reference FGMRES+GemslrClass (oracle/_ref), {threads} single-threaded processes at once, each "
                  f"its own setup and {solves} full {GRID[0]}^3 solves ({r['iters']} iterations each) of which the "
                  f"last {args.steps} are timed; solves/s summed over the processes")
    else:
        r, why = reference_run(threads, solves, dump=False)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        timed = r["times"][args.warmup:]
        t_solve = statistics.mean(timed)
        value = 1.0 / t_solve
        timed_s = sum(timed)
        sample = (f"reference FGMRES+GemslrClass (oracle/_ref) on {threads} threads: {solves} full {GRID[0]}^3 "
                  f"solves ({r['iters']} iterations, true rel-res {r['true_rel_res']:.2e}) after one setup, the "
                  f"last {args.steps} timed")
    line = {
        "impl": "reference", "metric": metric_name(), "value": value, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_solve * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config("reference"),
        "detail": {"iters": r["iters"], "true_rel_res": r["true_rel_res"], "setup_s": r["setup_s"],
                   "ref_mode": args.ref_mode, "timed_s": timed_s, "wall_s": r["wall_s"]},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ GPU arm
def _batch(h, p, R, n, B_dev, X_dev, ev_a, ev_b):
    import torch
    X_dev.zero_()
    torch.cuda.synchronize()
    ev_a.record()
    res = h.solve_batch_ptr(R, X_dev.data_ptr(), n, B_dev.data_ptr(), n, LOCATION_DEVICE, p)
    ev_b.record()
    ev_b.synchronize()
    return res, ev_a.elapsed_time(ev_b)


def _fit_slots(h, R, lanes, basis_bytes_per_rhs):
    """Slots for R right-hand sides in flight.  Each holds its own Krylov basis (allocated at its first solve, so
    it is counted here against the device's free memory, with 4 GB to spare); on a GPU with less free memory the
    batch shrinks until the slots fit.  Returns (R, nslots)."""
    import torch
    from pargemslr_b200._abi import ERROR_OOM, PgxError
    while True:
        nslots = 1 + -(-(R - 1) // lanes)
        try:
            h.set_slots(nslots)
        except PgxError as exc:
            if exc.code != ERROR_OOM or R <= lanes:
                raise
            h.set_slots(1)
            R = max(lanes, R - 4 * lanes)
            continue
        free, _ = torch.cuda.mem_get_info()
        pending = (1 + (nslots - 1) * lanes) * basis_bytes_per_rhs
        if pending + (4 << 30) <= free or R <= lanes:
            return R, nslots
        h.set_slots(1)
        R = max(lanes, R - 4 * lanes)


def _fp64_comparison(args, st, A, p, n, R, kdim, B_dev, X_dev, ev_a, ev_b, device):
    """The FP64 preconditioner on the same setup and right-hand sides: one solve at a time, and batched like the
    headline (as many right-hand sides in flight as fit)."""
    import torch
    from pargemslr_b200.handle import GemslrHandle
    h64 = (GemslrHandle(st, precision="fp64", device=device) if st is not None
           else GemslrHandle.from_matrix(A, p, precision="fp64", device=device))
    try:
        pm, pit = [], []
        for k in range(3):
            x1 = torch.zeros(n, dtype=torch.float64, device=B_dev.device)
            torch.cuda.synchronize()
            ev_a.record()
            r1 = h64.solve_device(x1.data_ptr(), B_dev[k % R].data_ptr(), params=p)
            ev_b.record()
            ev_b.synchronize()
            if k > 0:  # the first solve is warm-up
                pm.append(ev_a.elapsed_time(ev_b))
                pit.append(r1["iters"])
        plain = {"solves_per_s": len(pm) / (sum(pm) / 1e3), "ms_per_solve": sum(pm) / len(pm), "iters": pit,
                 "what": "FP64 preconditioner, one solve at a time (pgx_gemslr_solve), same setup and RHS"}
        h64.set_lanes(args.lanes)
        R64, ns64 = _fit_slots(h64, R, args.lanes, n * (kdim + 1) * 16)
        B64, X64 = B_dev[:R64], X_dev[:R64]
        _batch(h64, p, R64, n, B64, X64, ev_a, ev_b)  # warm-up
        bm, bit = [], []
        for _ in range(2):
            res64, t_ms = _batch(h64, p, R64, n, B64, X64, ev_a, ev_b)
            bm.append(t_ms)
            bit.extend(r["iters"] for r in res64)
        batched = {"solves_per_s": 2 * R64 / (sum(bm) / 1e3), "solves_per_step": R64, "slots": ns64,
                   "lanes_per_slot": args.lanes, "iters": [min(bit), max(bit)],
                   "what": "FP64 preconditioner, batched like the headline (pgx_gemslr_solve_batch); the width is "
                           "the headline's unless its Krylov bases (8+8 bytes per entry) do not fit"}
        return plain, batched
    finally:
        h64.close()


def run_pgx(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.structures import from_dump

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    p = P.workload_params(WORKLOAD)
    if args.local_order == "multicolor":
        if args.setup != "own":
            raise SystemExit("--local-order multicolor needs --setup own (the reference's setup orders by RCM)")
        p[P.ILU_PERM_OPTION_GLOBAL] = p[P.ILU_PERM_OPTION_LOCAL] = P.REORDER_MULTICOLOR
    A, n, _, _ = build_problem()
    threads = os.cpu_count() or 1

    # --- setup (untimed) and the reference's own solve of the first right-hand side
    t0 = time.time()
    ref, ref_why, st = None, None, None
    if args.setup == "reference":
        ref, ref_why = reference_run(threads, 1, dump=True)
        if ref is None:
            raise SystemExit("--setup reference: " + ref_why)
        log("reference setup and solve: %.1f s (%d iterations)" % (ref["wall_s"], ref["iters"]))
        st = from_dump(os.path.join(ref["dir"], "setup.bin"))
        h = GemslrHandle(st, precision=args.precision, device=local)
    elif args.setup == "parallel":
        from pargemslr_b200.structures import from_parallel_dump
        ref, ref_why = reference_run_parallel_class(threads)
        if ref is None:
            raise SystemExit("--setup parallel: " + ref_why)
        log("reference ParallelGemslrClass setup and solve: %.1f s (%d iterations)" % (ref["wall_s"], ref["iters"]))
        st = from_parallel_dump(os.path.join(ref["dir"], "setup_par.bin"))
        h = GemslrHandle(st, precision=args.precision, device=local)
    else:
        h = GemslrHandle.from_matrix(A, p, precision=args.precision, device=local)
    setup_s = time.time() - t0
    log("handle committed")

    R = args.batch
    xts = np.stack([problems.x_true(n, SEED + r) for r in range(R)])
    B = np.stack([problems.spmv(A, xts[r]) for r in range(R)])
    if ref is not None:
        # right-hand side 0 is the reference's own b (its MatVec of the same x_true)
        B[0] = pgxd.read(os.path.join(ref["dir"], "problem.bin"))["b"]
        x_ref = pgxd.read(os.path.join(ref["dir"], "solution.bin"))["x"]
    kdim = int(p[P.SOLVER_KDIM])
    h.set_lanes(args.lanes)
    R, nslots = _fit_slots(h, R, args.lanes, n * (kdim + 1) * (8 + (4 if args.precision == "mixed" else 8)))
    xts, B = xts[:R], B[:R]
    B_dev = torch.from_numpy(B).to(dev)
    X_dev = torch.zeros_like(B_dev)
    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)

    log("%d right-hand sides in %d slots" % (R, nslots))
    for _ in range(args.warmup):
        _batch(h, p, R, n, B_dev, X_dev, ev_a, ev_b)
    log("warm-up done")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    wall0 = time.perf_counter()
    ms, iters, rel, launches, lat = [], [], [], [], []
    first = None
    torch.cuda.nvtx.range_push("timed")  # lets a profiler capture the timed region alone
    for _ in range(args.steps):
        res, t_ms = _batch(h, p, R, n, B_dev, X_dev, ev_a, ev_b)
        ms.append(t_ms)
        lat.extend(r["solve_ms"] for r in res)
        iters.extend(r["iters"] for r in res)
        rel.extend(r["true_rel_res"] for r in res)
        launches.append(sum(r["launches"] for r in res))
        first = res[0]
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    total_ms = max_over_ranks(sum(ms), dev)
    if world > 1:
        dist.barrier()
    value = world * args.steps * R / (total_ms / 1e3)
    X = X_dev.cpu().numpy()
    x_err = max(float(np.linalg.norm(X[r] - xts[r]) / np.linalg.norm(xts[r])) for r in range(1, R)) if R > 1 else None
    parity = None
    if ref is not None:
        dref = float(np.linalg.norm(X[0] - x_ref) / np.linalg.norm(x_ref))
        parity = {"what": "right-hand side 0 (the reference's b) against the reference's own FP64 CPU solve on "
                          "the same imported setup",
                  "iters": first["iters"], "iters_ref": ref["iters"], "true_rel_res": first["true_rel_res"],
                  "true_rel_res_ref": ref["true_rel_res"], "x_vs_x_ref": dref,
                  "iters_bar": ("+-1" if args.precision == "fp64" else "<= +15%"),
                  "ok": bool(dref <= 1e-6 and first["true_rel_res"] <= 1e-8 and
                             (abs(first["iters"] - ref["iters"]) <= 1 if args.precision == "fp64"
                              else first["iters"] <= int(np.floor(1.15 * ref["iters"])) + 1))}

    # end to end through the host-buffer C ABI call: pinned host B and X, the
    # copies in and out are inside every timed call
    B_host = torch.from_numpy(B).pin_memory()
    X_host = torch.zeros((R, n), dtype=torch.float64).pin_memory()
    e2e_ms = []
    e2e_steps = min(args.steps, 5)
    for _ in range(e2e_steps):
        X_host.zero_()
        torch.cuda.synchronize()
        ev_a.record()
        h.solve_batch_ptr(R, X_host.data_ptr(), n, B_host.data_ptr(), n, LOCATION_HOST, p)
        ev_b.record()
        ev_b.synchronize()
        e2e_ms.append(ev_a.elapsed_time(ev_b))
    e2e_total = max_over_ranks(sum(e2e_ms) / 1e3, dev)
    log("timed and e2e steps done: %.3f s per step" % (total_ms / args.steps / 1e3))

    # roofline of the dominant kernel: the level-0 triangular passes, merged over
    # the lanes of a multi-lane slot (the kernel the batch spends its time in)
    torch.cuda.nvtx.range_push("kernel_stats")  # plain stream launches, outside any graph
    if args.lanes > 1:
        blo_ms, blo_bytes = h.kernel_stats(3, 0, reps=5)
        bup_ms, bup_bytes = h.kernel_stats(4, 0, reps=5)
    lo_ms, lo_bytes = h.kernel_stats(0, 0, reps=5)
    up_ms, up_bytes = h.kernel_stats(1, 0, reps=5)
    spmv_ms, spmv_bytes = h.kernel_stats(2, 0, reps=5)
    torch.cuda.nvtx.range_pop()
    h.set_slots(1)
    h.set_lanes(1)
    h.close()
    del B_host, X_host

    # the FP64 preconditioner on the same setup: batched at the same width (as
    # many right-hand sides as fit), and one solve at a time
    fp64_batched, plain, fp64_error = None, None, None
    if world == 1 and not args.no_fp64 and args.precision == "mixed":
        try:
            plain, fp64_batched = _fp64_comparison(args, st, A, p, n, R, kdim, B_dev, X_dev, ev_a, ev_b, local)
        except Exception as exc:  # the headline line is printed regardless
            fp64_error = repr(exc)[:300]

    peak, peak_kind = measured_peak_hbm()
    single = {"bytes_per_launch": (lo_bytes + up_bytes) / 2.0, "ms_per_launch": (lo_ms + up_ms) / 2.0}
    single["achieved"] = single["bytes_per_launch"] / (single["ms_per_launch"] * 1e-3) / 1e9
    if args.lanes > 1:
        kname = ("trsv_pipe_kernel (level-0 ILU L and U passes merged over %d lanes, mean; one CTA per "
                 "subdomain)" % args.lanes)
        tri_bytes = (blo_bytes + bup_bytes) / 2.0
        tri_ms = (blo_ms + bup_ms) / 2.0
    else:
        kname = "trsv_pipe_kernel (level-0 ILU L and U passes, mean; one CTA per subdomain)"
        tri_bytes, tri_ms = single["bytes_per_launch"], single["ms_per_launch"]
    achieved = tri_bytes / (tri_ms * 1e-3) / 1e9
    traffic = ncu_traffic(args.lanes)
    detail = {"precision": args.precision, "setup_kind": args.setup, "local_order": args.local_order,
              "solves_per_step": R, "slots": nslots, "lanes_per_slot": args.lanes, "setup_s": round(setup_s, 2),
              "iters": [min(iters), max(iters)], "true_rel_res_max": max(rel),
              "x_err_max_vs_x_true": x_err, "parity_vs_reference": parity,
              "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                             "what": "device time of each solve inside the batch (its slot's events)"},
              "fp64_plain": plain, "fp64_batched": fp64_batched, "fp64_error": fp64_error,
              "mixed_over_fp64_batched": (value / fp64_batched["solves_per_s"]) if fp64_batched else None,
              "mixed_over_fp64_plain": (value / plain["solves_per_s"]) if plain else None,
              "l2": "inputs larger than L2 (level-0 factors alone are about 1 GB)",
              "host_wall_s": wall, "e2e_steps": e2e_steps}
    line = {
        "metric": metric_name(), "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 preconditioner / f64 FGMRES" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": workload_config(args.setup),
        "detail": detail,
        "e2e": {"value": world * e2e_steps * R / e2e_total, "unit": "solves/s", "h2d_bytes_per_step": 16 * n * R,
                "d2h_bytes_per_step": 8 * n * R},
        "gpu_launches": int(sum(launches)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": kname, "single_lane": single,
                     "bytes_per_launch": tri_bytes, "ms_per_launch": tri_ms,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None,
                     "traffic_source": traffic.get("how") if traffic else None,
                     "spmv": {"achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "ms": spmv_ms}},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and GRID == (128, 128, 128):
        cpu = ref
        if cpu is None:
            cpu, _ = reference_run(threads, 1, dump=False)
        if cpu is None:
            line["cpu_baseline"] = None
        else:
            line["cpu_baseline"] = {
                "value": 1.0 / cpu["times"][-1], "unit": "solves/s", "cores": threads, "kind": "reference",
                "sample": f"reference CPU solver (oracle/_ref) on {threads} threads: one full solve of the first "
                          f"right-hand side ({cpu['iters']} FGMRES iterations, true rel-res "
                          f"{cpu['true_rel_res']:.2e}); its setup ({cpu['setup_s']:.1f} s) untimed"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_serve(args):
    """Serving workload: a Poisson stream of requests over resident preconditioned matrices (pgx_pool_*).

    `--serve-matrices` random nonsymmetric sparse systems with rows log-uniform in [--serve-rows-min,
    --serve-rows-max] (7-27 nonzeros per row, off-diagonals N(0,1), diagonal 1.2 x the row's absolute off-diagonal
    sum), each set up once (untimed) and kept resident; one pool with a device-memory budget of 90% of the free
    memory admits requests by the bytes of their slot (work space and FGMRES(40) Krylov basis).  For every arrival
    rate, --serve-requests requests arrive with exponential gaps, each for a matrix drawn uniformly with a seeded
    U[-1,1] right-hand side (a few per matrix, reused), solved to rel-res 1e-8.  An untimed burst of --serve-warmup
    requests first brings the pool to its working set of slots.  Latency is arrival to collection on
    the host clock; throughput is requests finished over the span from the first arrival to the last finish."""
    import torch
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.serving import Pool

    rng = np.random.default_rng(2026)
    p = P.workload_params("serve")
    lo, hi = args.serve_rows_min, args.serve_rows_max
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), size=args.serve_matrices)).astype(int)
    hs, setup_s = [], 0.0
    for i, n in enumerate(sizes):
        A = problems.random_diag_dominant(int(n), 1000 + i)
        t0 = time.time()
        hs.append(GemslrHandle.from_matrix(A, p, precision=args.precision))
        setup_s += time.time() - t0
        log("matrix %d: n=%d set up" % (i, n))
    free, _ = torch.cuda.mem_get_info()
    budget = int(0.9 * free)
    pool = Pool(budget, p)
    for h in hs:
        pool.add(h)
    rhs_per = 4
    B = [[torch.from_numpy(np.random.default_rng(7 * i + k).uniform(-1, 1, h.n)).cuda() for k in range(rhs_per)]
         for i, h in enumerate(hs)]
    pool.start()
    rid = 0
    # warm-up, untimed: one burst of --serve-warmup requests spread over the members, submitted together, so the
    # slots (and their captured restart graphs) that the measured rates will use exist before any latency counts
    if args.serve_warmup > 0:
        t0 = time.time()
        pending, warm_x = set(), []
        for k in range(args.serve_warmup):
            m = k % len(hs)
            xs_w = torch.zeros(hs[m].n, dtype=torch.float64, device="cuda")
            pool.submit_ptr(m, xs_w.data_ptr(), B[m][k % rhs_per].data_ptr(), LOCATION_DEVICE, rid)
            pending.add(rid)
            rid += 1
            warm_x.append(xs_w)
        while pending:
            for i, _ in pool.collect():
                pending.discard(i)
            time.sleep(0.0005)
        warm_x.clear()
        log("warm-up: %d requests, %d slots, %.1f s" % (args.serve_warmup, pool.stats()["slots"], time.time() - t0))
    results = []
    for rate in args.serve_rates:
        gaps = rng.exponential(1.0 / rate, size=args.serve_requests)
        members = rng.integers(0, len(hs), size=args.serve_requests)
        arrivals = {}
        xs = {}
        lat, iters, ok = [], [], 0
        t_start = time.perf_counter()
        t_next = t_start
        k = 0
        last_done = t_start
        while k < args.serve_requests or len(arrivals) > 0:
            now = time.perf_counter()
            while k < args.serve_requests and t_next <= now:
                m = int(members[k])
                xs[rid] = torch.zeros(hs[m].n, dtype=torch.float64, device="cuda")
                pool.submit_ptr(m, xs[rid].data_ptr(), B[m][k % rhs_per].data_ptr(), LOCATION_DEVICE, rid)
                arrivals[rid] = t_next
                rid += 1
                k += 1
                if k < args.serve_requests:
                    t_next += gaps[k]
            for i, r in pool.collect():
                t = time.perf_counter()
                lat.append((t - arrivals.pop(i)) * 1e3)
                iters.append(r["iters"])
                ok += int(r["status"] == 0 and r["true_rel_res"] <= 1e-8)
                xs.pop(i, None)
                last_done = t
            time.sleep(0.0002)
        span = last_done - t_start
        st = pool.stats()
        results.append({"rate_per_s": rate, "requests": args.serve_requests, "solves_per_s": len(lat) / span,
                        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                        "iters_mean": float(np.mean(iters)), "converged": ok, "slots": st["slots"],
                        "peak_bytes": st["peak_bytes"]})
        log("rate %s: %.1f solves/s p50 %.1f ms p99 %.1f ms" % (rate, results[-1]["solves_per_s"],
                                                                results[-1]["p50_ms"], results[-1]["p99_ms"]))
    pool.stop()
    pool.close()
    for h in hs:
        h.close()
    line = {"metric": "serving: solves/s and p50/p99 request latency under Poisson arrivals, rel-res 1e-8",
            "unit": "solves/s", "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
            "dtype": "f32 preconditioner / f64 FGMRES" if args.precision == "mixed" else "f64",
            "config": {"workload": "%d random nonsymmetric sparse systems, rows log-uniform in [%d, %d], 7-27 "
                                   "nonzeros per row, 2 levels, ILUT 1e-2/20, rank 8, FGMRES(40) to 1e-8"
                                   % (len(hs), lo, hi),
                       "budget_bytes": budget, "setup_s": round(setup_s, 1), "warmup_requests": args.serve_warmup, "rows": [int(v) for v in sizes]},
            "value": max(r["solves_per_s"] for r in results), "rates": results}
    print(json.dumps(line), flush=True)


def run_uneven(args):
    """Batched uneven systems: --systems upwind convection-diffusion problems -Laplace(u) + beta . grad(u) on n x n
    grids, n log-uniform in [32, 512] and beta ~ U[0, 50]^2 (seeded), b ~ U[-1, 1]; 2 levels, ILUT 1e-2/20, rank 8,
    inner Schur FGMRES(5), FGMRES(30) to rel-res 1e-8 from x0 = 0.  Each system is set up once by this library's
    host setup (untimed) and all of them are packed into one pgx_systems object; a step solves every system with ONE
    persistent kernel launch under the schedule the autotuner picked.  value: systems per second of device time of
    that launch (inputs resident); e2e: the same solves from and to host arrays, copies inside the timed region.
    Compared with each system solved by its own handle (pgx_gemslr_solve, one after another) on a sample, and with
    the reference CPU solver (its own setup, single-threaded processes, one per host thread) on a sample."""
    import torch
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.systems import SystemsBatch, shard_systems

    # several GPUs (torchrun): the systems are split by estimated cost, each rank solves its share in one launch of
    # its own, and the timed regions are reduced to their maximum over ranks; no data crosses GPUs
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=1800))
    count = args.systems
    rng = np.random.default_rng(SEED + 4)
    grid = np.exp(rng.uniform(np.log(32), np.log(args.uneven_nmax), size=count)).astype(int)
    beta = rng.uniform(0.0, 50.0, size=(count, 2))
    mine = shard_systems([float(g) ** 3 for g in grid], world)[rank]  # cost ~ n^1.5, n = g^2
    mine_set = set(mine)
    p = P.workload_params("convdiff")
    mats, B, hs = [], [], []
    t0 = time.time()
    for k in range(count):
        g = int(grid[k])
        b = rng.uniform(-1.0, 1.0, g * g)  # drawn for every system so the stream is the same on every rank
        if k not in mine_set:
            continue
        A = problems.upwind_convdiff_2d(g, g, float(beta[k, 0]), float(beta[k, 1]))
        mats.append(A)
        B.append(b)
        hs.append(GemslrHandle.from_matrix(A, p, precision=args.precision, device=local))
        if len(hs) % 64 == 0:
            log("set up %d/%d systems (%.1f s)" % (len(hs), len(mine), time.time() - t0))
    setup_s = time.time() - t0
    total = count
    count = len(mine)
    sizes = np.array([int(grid[k]) ** 2 for k in mine])
    unknowns = int(sum(int(g) ** 2 for g in grid))
    sb = SystemsBatch(hs)
    t0 = time.time()
    best = sb.tune(B, params=p, stride=args.uneven_tune_stride)
    table = sb.tune_table()
    log("autotuner on every %d-th system: %s in %.1f ms (%.1f s for %d candidates)"
        % (args.uneven_tune_stride, sb.schedule, best, time.time() - t0, len(table)))
    # device-resident inputs: b and x0 = 0 on the GPU
    bd = [torch.from_numpy(b).cuda(local) for b in B]
    xflat = torch.zeros(int(sizes.sum()), dtype=torch.float64, device="cuda:%d" % local)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    xptr = [xflat[offs[k]:offs[k + 1]].data_ptr() for k in range(count)]
    bptr = [b.data_ptr() for b in bd]
    clocks = ClockSampler(local)
    R = None
    for _ in range(args.warmup):
        xflat.zero_()
        torch.cuda.synchronize()
        R = sb.solve_ptrs(xptr, bptr, LOCATION_DEVICE, params=p)
    ms = []
    clocks.start()
    for _ in range(args.steps):
        xflat.zero_()
        torch.cuda.synchronize()
        R = sb.solve_ptrs(xptr, bptr, LOCATION_DEVICE, params=p)
        ms.append(sb.last_launch_ms())
    clk = clocks.stop()
    ms_step = max_over_ranks(max(ms), "cuda")
    iters = np.array([r["iters"] for r in R])
    trr = np.array([r["true_rel_res"] for r in R])
    ok = int(np.sum([(r["status"] == 0 and r["true_rel_res"] <= 1e-8) for r in R]))
    ts, te, ttri = sb.timing()
    span = te - ts
    slow = int(np.argmax(span))
    # end to end from host arrays
    e2e_s = []
    for _ in range(args.steps):
        if world > 1:
            dist.barrier()
        t1 = time.perf_counter()
        X, Rh = sb.solve(B, params=p)
        e2e_s.append(time.perf_counter() - t1)
    e2e = total / max_over_ranks(max(e2e_s), "cuda")
    h2d = unknowns * 8 * 2
    d2h = unknowns * 8
    # each system by its own handle, one after another, on a sample spanning the sizes
    order = np.argsort(sizes)
    per_handle = None
    if args.uneven_sample > 0 and world == 1:
        sample = order[:: max(1, count // args.uneven_sample)]
        t_one = []
        it_one = []
        for k in sample:
            xs, rs = hs[k].solve(B[k], params=p)
            t_one.append(rs["solve_ms"] * 1e-3)
            it_one.append(rs["iters"])
        scale = float(sizes.sum()) / float(sizes[sample].sum())
        per_handle = {"systems_per_s": count / (sum(t_one) * scale), "sample": int(len(sample)), "iters": it_one,
                      "what": "each system by its own handle (pgx_gemslr_solve: per-kernel launches and a graph "
                              "per restart cycle), one after another; device time summed over every %d-th system by "
                              "size, scaled by total over sampled unknowns" % max(1, count // args.uneven_sample)}
    # the reference CPU solver (its own setup) on a sample, one single-threaded process per host thread
    ref = None
    drv = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver")
    if os.path.exists(drv) and not args.no_cpu_baseline and world == 1:
        from concurrent.futures import ThreadPoolExecutor
        threads = os.cpu_count() or 1
        rsample = order[:: max(1, count // args.uneven_ref_sample)]

        def one(k):
            d = tempfile.mkdtemp(prefix="pgx_uneven_")
            A = mats[k]
            f = os.path.join(d, "A.bin")
            pgxd.write(f, {"A.i": A[0].astype(np.int32), "A.j": A[1].astype(np.int32),
                           "A.a": A[2].astype(np.float64)})
            rf = os.path.join(d, "rhs.bin")
            pgxd.write(rf, {"b": B[k]})
            cmd = [drv, "--out", d, "--csr", f, "--rhs", rf, "--solve", "--threads", "1"]
            for i, v in enumerate(p):
                cmd += ["--param", f"{i}={float(v)!r}"]
            subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL,
                           env=dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1"))
            r = {}
            with open(os.path.join(d, "result.txt")) as fh:
                for line in fh:
                    key, v = line.strip().split("=", 1)
                    r[key] = v
            x_ref = pgxd.read(os.path.join(d, "solution.bin"))["x"]
            return k, float(r["solve_s"]), float(r["setup_s"]), int(r["iters"]), x_ref

        t1 = time.time()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            outs = list(ex.map(one, rsample))
        wall = time.time() - t1
        rscale = float(sizes.sum()) / float(sizes[rsample].sum())
        solve_sum = sum(o[1] for o in outs)
        xerr = [float(np.linalg.norm(X[k] - xr) / np.linalg.norm(xr)) for k, _, _, _, xr in outs]
        ref = {"systems_per_s": count / (solve_sum * rscale / threads), "threads": threads,
               "sample": int(len(rsample)), "solve_s_sum": solve_sum, "setup_s_sum": sum(o[2] for o in outs),
               "wall_s": wall, "iters": [o[3] for o in outs], "iters_gpu": [int(iters[k]) for k in rsample],
               "x_vs_x_ref_max": max(xerr),
               "what": "reference CPU solver (oracle/_ref) with its own setup, one single-threaded process per host "
                       "thread, every %d-th system by size; solve time summed over the sample, scaled by total "
                       "unknowns over sampled unknowns, divided by the threads" % max(1, count // args.uneven_ref_sample)}
        log("reference sample: %d systems, %.1f s of solves" % (len(rsample), solve_sum))
    line = {
        "metric": "systems/s (batched uneven GeMSLR-FGMRES(30), rel-res 1e-8, %d systems in one launch per GPU)"
                  % total,
        "value": total / (ms_step * 1e-3), "unit": "systems/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32 preconditioner / f64 FGMRES" if args.precision == "mixed" else "f64",
        "data": "synthetic",
        "config": {"workload": "%d upwind convection-diffusion systems -Lu + beta.grad u on n x n grids, n "
                               "log-uniform in [32, %d], beta ~ U[0,50]^2, b ~ U[-1,1], 2 levels, ILUT 1e-2/20, "
                               "rank 8, inner Schur FGMRES(5), FGMRES(30) to rel-res 1e-8 from x0 = 0"
                               % (total, args.uneven_nmax),
                   "unknowns": unknowns, "setup": "this library's host setup per system, untimed",
                   "sharding": "by estimated cost over %d GPU(s), no exchange" % world,
                   "schedule": {"threads": sb.schedule[0], "ctas_per_sm": sb.schedule[1], "spmv_lanes": sb.schedule[2],
                                "prefetch_levels": sb.schedule[3]},
                   "l2": "inputs larger than L2 (%.1f GB of packed structures and Krylov bases)"
                         % (sb.device_bytes() / 1e9)},
        "e2e": {"value": e2e, "unit": "systems/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": 1,
        "detail": {"converged": ok, "iters_min": int(iters.min()), "iters_max": int(iters.max()),
                   "iters_mean": float(iters.mean()), "true_rel_res_max": float(trr.max()),
                   "setup_s": round(setup_s, 1), "tune_table": table,
                   "system_ms": {"p50": float(np.percentile(span, 50)), "p99": float(np.percentile(span, 99)),
                                 "max": float(span.max()), "last_end": float(te.max()),
                                 "sum": float(span.sum()), "triangular_share": float(ttri.sum() / span.sum()),
                                 "slowest": {"n": int(sizes[slow]), "iters": int(iters[slow]), "ms": float(span[slow]),
                                             "triangular_ms": float(ttri[slow])}},
                   "per_handle": per_handle,
                   "reference": ref},
        "clocks": clk,
    }
    if ref:
        line["cpu_baseline"] = {"value": ref["systems_per_s"], "unit": "systems/s", "cores": ref["threads"],
                                "kind": "reference", "sample": ref["what"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    sb.close()
    for h in hs:
        h.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_complex(args):
    """The complex workload: a 96^3 7-point Laplacian shifted by -(0.05 + 0.01i) (indefinite), the reference's
    complexd GemslrClass setup (5 levels, ILUT 1e-3, rank 32), FGMRES(100) to rel-res 1e-8, and 16 seeded
    complex-Gaussian right-hand sides solved as one block in a 16-lane slot (triangular passes merged four lanes
    at a time; with the complex64 preconditioner every low-rank correction is one tcgen05 GEMM pair for all 16).
    The reference solves the first --ref-rhs of them one at a time on all host threads (its setup untimed); the
    GPU arm reports both preconditioner precisions."""
    import torch
    from pargemslr_b200.handle import GemslrHandle
    from pargemslr_b200.structures import from_dump

    g = args.grid if args.grid != 128 else 96
    n = g ** 3
    nrhs = 16
    p = P.workload_params("zlap3d_96")
    rng = np.random.default_rng(SEED)
    Bc = rng.standard_normal((nrhs, n)) + 1j * rng.standard_normal((nrhs, n))
    threads = os.cpu_count() or 1
    d = tempfile.mkdtemp(prefix="pgx_zref_")
    rf = os.path.join(d, "rhs.bin")
    kref = max(1, min(args.ref_rhs, nrhs))
    pgxd.write(rf, {"B": np.ascontiguousarray(Bc[:kref]).view(np.float64).ravel(), "nrhs": np.array([kref], np.int32)})
    drv = os.path.join(ROOT, "oracle", "_ref", "pgx_ref_driver_z")
    if not os.path.exists(drv):
        raise SystemExit("oracle/_ref/pgx_ref_driver_z not built")
    cmd = [drv, "--out", d, "--lap", str(g), str(g), str(g), "0.05", "0.01", "0", "0", "0", "--rhs", rf, "--dump",
           "--solve", "--threads", str(threads)]
    for i, v in enumerate(p):
        cmd += ["--param", f"{i}={float(v)!r}"]
    t0 = time.time()
    subprocess.run(cmd, check=True, env=dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1"),
                   stdout=subprocess.DEVNULL)
    log("complex reference setup and %d solves: %.1f s" % (kref, time.time() - t0))
    res_ref = dict(line.strip().split("=", 1) for line in open(os.path.join(d, "result.txt")))
    it_ref = [int(t) for t in res_ref["iters"].split(",")]
    t_ref = [float(t) for t in res_ref["solve_times"].split(",")]
    sol = pgxd.read(os.path.join(d, "solution.bin"))
    x_ref = [sol["x%d" % r].view(np.complex128) for r in range(kref)]
    st = from_dump(os.path.join(d, "setup.bin"))
    dev = torch.device("cuda", 0)
    Bd = torch.from_numpy(np.ascontiguousarray(Bc)).to(dev)
    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)
    out = {}
    for precision in ("mixed", "fp64"):
        h = GemslrHandle(st, precision=precision, device=0)
        try:
            h.set_lanes(nrhs)
            h.set_slots(2)
            Xd = torch.zeros_like(Bd)
            Bf = Bd.view(torch.float64)
            Xf = Xd.view(torch.float64)
            ms, its, rel = [], [], []
            for step in range(args.warmup + args.steps):
                Xd.zero_()
                torch.cuda.synchronize()
                ev_a.record()
                res = h.solve_batch_ptr(nrhs, Xf.data_ptr(), n, Bf.data_ptr(), n, LOCATION_DEVICE, p)
                ev_b.record()
                ev_b.synchronize()
                if step >= args.warmup:
                    ms.append(ev_a.elapsed_time(ev_b))
                    its.extend(r["iters"] for r in res)
                    rel.extend(r["true_rel_res"] for r in res)
            X = Xd.cpu().numpy()
            dx = [float(np.linalg.norm(X[r] - x_ref[r]) / np.linalg.norm(x_ref[r])) for r in range(kref)]
            out[precision] = {"solves_per_s": nrhs * len(ms) / (sum(ms) / 1e3), "ms_per_block": sum(ms) / len(ms),
                              "iters": [min(its), max(its)], "true_rel_res_max": max(rel),
                              "x_vs_x_ref": dx, "iters_first": [res[r]["iters"] for r in range(kref)]}
            log("%s: %.2f solves/s, iterations %s" % (precision, out[precision]["solves_per_s"],
                                                       out[precision]["iters"]))
        finally:
            h.set_lanes(1)
            h.close()
    mixed = out["mixed"]
    ok = all(v <= 1e-6 for v in out["fp64"]["x_vs_x_ref"]) and \
        all(abs(a - b) <= 1 for a, b in zip(out["fp64"]["iters_first"], it_ref)) and \
        all(a <= int(np.floor(1.15 * b)) + 1 for a, b in zip(mixed["iters_first"], it_ref))
    line = {
        "metric": "solves/s (GeMSLR-FGMRES(100), rel-res 1e-8, complex shifted 3D Laplacian %d^3, 16-RHS block)" % g,
        "value": mixed["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed["ms_per_block"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64 preconditioner / c128 FGMRES", "data": "synthetic",
        "config": {"workload": "complex shifted 3D 7-point Laplacian %d^3 (n=%d), shift 0.05+0.01i, 5 levels, ILUT "
                               "1e-3, rank 32, inner Schur FGMRES(5), FGMRES(100) to 1e-8 from x0 = 0, 16 seeded "
                               "complex-Gaussian right-hand sides as one 16-lane block" % (g, n),
                   "setup": "the reference's complexd GemslrClass::Setup (oracle/_ref/pgx_ref_driver_z), untimed"},
        "detail": {"mixed": mixed, "fp64": out["fp64"], "mixed_over_fp64": mixed["solves_per_s"] /
                   out["fp64"]["solves_per_s"],
                   "reference": {"iters": it_ref, "solve_s": t_ref, "threads": threads,
                                 "solves_per_s": len(t_ref) / sum(t_ref)},
                   "parity_ok": bool(ok)},
        "cpu_baseline": {"value": len(t_ref) / sum(t_ref), "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": "reference complex FGMRES+GemslrClass (oracle/_ref/pgx_ref_driver_z) on %d threads, "
                                   "the first %d right-hand sides one at a time" % (threads, kref)},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["pgx", "reference"], default="pgx")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--setup", choices=["reference", "parallel", "own"], default="reference",
                    help="whose setup builds the preconditioner: the reference's GemslrClass::Setup, imported through "
                         "the C ABI (default); the reference's ParallelGemslrClass::Setup at one rank, its per-level "
                         "permutations composed; or this library's host setup")
    ap.add_argument("--batch", type=int, default=96, help="right-hand sides solved concurrently per step")
    ap.add_argument("--lanes", type=int, default=4, choices=[1, 2, 4],
                    help="right-hand sides each slot advances in lockstep")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-preconditioner comparison solves")
    ap.add_argument("--local-order", choices=["rcm", "multicolor"], default="rcm",
                    help="order inside subdomains for this library's setup (--setup own): reverse Cuthill-McKee "
                         "(the reference's option) or multicolor (red-black on this grid)")
    ap.add_argument("--ref-mode", choices=["latency", "throughput"], default="latency",
                    help="reference arm: one process on all host threads (latency), or one single-threaded "
                         "process per host thread at once (throughput)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=128,
                    help="cube edge of the Laplacian (128 is the headline workload; smaller grids for profiling)")
    ap.add_argument("--workload", choices=["laplacian", "serve", "complex", "uneven"], default="laplacian",
                    help="laplacian: the headline batch benchmark; serve: Poisson arrivals over resident matrices; "
                         "complex: 16 right-hand sides of the complex shifted 96^3 Laplacian as one block")
    ap.add_argument("--ref-rhs", type=int, default=2, help="complex workload: right-hand sides the reference solves")
    ap.add_argument("--systems", type=int, default=512, help="uneven workload: number of systems")
    ap.add_argument("--uneven-sample", type=int, default=32, help="uneven workload: systems solved by their own handle")
    ap.add_argument("--uneven-ref-sample", type=int, default=32,
                    help="uneven workload: systems the reference CPU solver solves")
    ap.add_argument("--uneven-nmax", type=int, default=512,
                    help="uneven workload: largest grid edge (512 is the workload; smaller for profiling)")
    ap.add_argument("--uneven-tune-stride", type=int, default=4,
                    help="uneven workload: the autotuner times every k-th system of the work list")
    ap.add_argument("--serve-matrices", type=int, default=64)
    ap.add_argument("--serve-rows-min", type=int, default=200000)
    ap.add_argument("--serve-rows-max", type=int, default=2000000)
    ap.add_argument("--serve-requests", type=int, default=2000, help="requests per arrival rate")
    ap.add_argument("--serve-warmup", type=int, default=256, help="untimed burst of requests before the rates")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[50, 200, 500, 1000, 2000])
    args = ap.parse_args()
    global GRID
    GRID = (args.grid,) * 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.workload == "complex":
        run_complex(args)
    elif args.workload == "uneven":
        run_uneven(args)
    else:
        run_pgx(args)


if __name__ == "__main__":
    main()
