"""Solve-phase benchmark: PCG solves/s on the 3D 7-point 128^3 high-contrast
SDDM grid (n = 2,097,152), tol 1e-8, FP64-verified.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm: one step = one PCG solve of one N(0,1) right-hand side through the
GPU-resident path (fp64 sweeps reproducing the reference arithmetic, fp64
SpMV / vectors). `value` times K device-resident solves with CUDA events on
the engine stream; `e2e` times the same solves through the public C ABI from
pinned host memory (b uploaded and x downloaded inside the timed region).
The roofline is the sweep kernel's: algorithmic bytes per sweep / measured
sweep time against the measured HBM copy bandwidth. The CPU baseline is the
reference's own cpu_solver (oracle/_ref) on the host cores, on a bounded
sample of the same solves.

--impl reference: the reference's CPU solve phase alone (rank 0), each step one
solve of the same system; prints the same JSON line with "impl": "reference".

With torchrun (N > 1) every rank solves its own replica (no collective on the
data path); value = all ranks' solves / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PCG solves/s (relres 1e-8, FP64-verified)"
GRID_N = 128
TOL = 1e-8
MAX_ITER = 500
FACTOR_SEED = 1
FACTOR_THREADS = 8


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def build_problem():
    from apxchol_b200 import gen, refsetup
    t0 = time.time()
    A = gen.grid3d(GRID_N, seed=1)
    t1 = time.time()
    F = refsetup.factorize(A, seed=FACTOR_SEED, threads=FACTOR_THREADS)
    t2 = time.time()
    log(f"[bench] grid3d_{GRID_N}: n={A.n} nnz(A)={A.nnz} gen {t1 - t0:.1f}s; factor nnz={F.nnz} "
        f"rounds={len(F.rounds)} factorize {t2 - t1:.1f}s")
    return A, F


def workload_config(A, F, info=None):
    cfg = {"workload": f"grid3d_{GRID_N} 7-point, weights 10^U[-3,3] (seed 1), boundary +1 (SDDM); "
                       f"plain FP64 PCG, 1 RHS/solve",
           "n": int(A.n), "nnz_A": int(A.nnz), "nnz_factor": int(F.nnz), "tol": TOL, "max_iter": MAX_ITER,
           "factor": f"apxchol factorize seed {FACTOR_SEED}, {FACTOR_THREADS} threads, block_greedy/vec_pool",
           "l2": "inputs larger than L2 (factor + operator > 400 MB per solve)"}
    if info is not None:
        cfg["nnz_stored"] = int(info.nnz_stored)
    return cfg


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(A, F, b, samples: int = 3):
    """The reference cpu_solver on this host (bounded sample of solves)."""
    import oracle
    if not oracle.ref_available():
        return None
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    R = oracle.Ref(A, F)
    times, its = [], []
    for _ in range(samples):
        x, it, res, secs = R.solve(b, TOL, MAX_ITER)
        times.append(secs)
        its.append(it)
    med = statistics.median(times)
    return {"value": 1.0 / med, "unit": "solves/s", "cores": cores, "kind": "reference",
            "sample": f"{samples} solves of the same 128^3 system (median {med * 1e3:.0f} ms, {its[0]} iterations), "
                      f"reference cpu_solver OMP_NUM_THREADS={cores}",
            "iterations": int(its[0])}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    from apxchol_b200 import gen
    A, F = build_problem()
    b = gen.rhs(A.n, 1000, False)
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return 0
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    R = oracle.Ref(A, F)
    for _ in range(args.warmup):
        R.solve(b, TOL, MAX_ITER)
    secs, its = [], []
    for _ in range(args.steps):
        x, it, res, s = R.solve(b, TOL, MAX_ITER)
        secs.append(s)
        its.append(it)
    total = sum(secs)
    v = args.steps / total
    tres = float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": workload_config(A, F), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} solves, reference cpu_solver OMP_NUM_THREADS={cores}"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "iterations": int(its[-1]), "true_relres": tres}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    from apxchol_b200 import gen, native

    torch.cuda.set_device(local_rank)
    A, F = build_problem()
    b = gen.rhs(A.n, 1000 + rank, False)
    eng = native.Engine(local_rank)
    t0 = time.time()
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    Op = native.DeviceOperator(eng, A, F.perm)
    log(f"[bench] upload factor+operator {time.time() - t0:.1f}s; stored nnz {D.info.nnz_stored}; "
        f"levels {D.info.fwd_levels}; device bytes {D.info.device_bytes / 1e6:.0f} MB")
    stream = torch.cuda.ExternalStream(eng.stream)
    n = A.n
    db = torch.from_numpy(b).cuda()
    dx = torch.empty(n, dtype=torch.float64, device="cuda")
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.empty(n, dtype=torch.float64).pin_memory()
    torch.cuda.synchronize()

    def solve_dev():
        _, r = native.pcg(eng, D, Op, db, dx, tol=TOL, max_iter=MAX_ITER, device_ptrs=True, true_residual=False)
        return r

    def solve_host():
        # host pointers (pinned): the library copies b in and x out inside the call
        r = native.PcgResult()
        native.check(eng.lib.apxb_pcg(eng.h, D.h, Op.h, hb.data_ptr(), hx.data_ptr(), TOL, MAX_ITER, 0, 0,
                                      native.ctypes.byref(r)))
        return r

    for _ in range(max(args.warmup, 3)):
        r = solve_dev()
    _, rv = native.pcg(eng, D, Op, db, dx, tol=TOL, max_iter=MAX_ITER, device_ptrs=True, true_residual=True)
    iters = rv.iterations
    x_host = dx.cpu().numpy()
    tres = float(np.linalg.norm(b - A.matvec(x_host)) / np.linalg.norm(b))
    log(f"[bench] rank {rank}: {iters} iterations, recurrence relres {rv.residual:.2e}, "
        f"fp64 true relres {tres:.2e} (device {rv.true_residual:.2e}), status {rv.status}")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- value: device-resident solves ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        ev0.record(stream)
        its = []
        for _ in range(args.steps):
            its.append(solve_dev().iterations)
        ev1.record(stream)
        barrier()
    dev_s = ev0.elapsed_time(ev1) * 1e-3
    # ---- e2e: host buffers through the C ABI ----
    for _ in range(2):
        solve_host()
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        solve_host()
    ev1.record(stream)
    barrier()
    e2e_s = ev0.elapsed_time(ev1) * 1e-3
    # ---- roofline: the sweep kernels ----
    dm = torch.from_numpy(np.random.default_rng(5).standard_normal(D.m)).cuda()
    dz = torch.empty_like(dm)
    torch.cuda.synchronize()
    D.sweep_pair_timed(dm, dz, 3)
    pair_s = D.sweep_pair_timed(dm, dz, 20)
    m, nnz_s = D.info.m, D.info.nnz_stored
    sweep_bytes = nnz_s * 8 + 4 * (m + 1) + 2 * m * 8
    sweep_s = pair_s / 2
    peak, peak_kind = measured_peak_hbm()
    achieved = sweep_bytes / sweep_s / 1e9
    # per-iteration algorithmic bytes (factor + matrix), and all traffic
    b_factor = 2 * (nnz_s * 8 + 4 * (m + 1))
    b_matrix = A.nnz * 12 + 4 * (n + 1)
    if world > 1:
        t = torch.tensor([dev_s, e2e_s], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_s, e2e_s = float(t[0]), float(t[1])
    if rank != 0:
        return 0
    launches_per_solve = 1 + 5 + 7 * iters + 2
    line = {
        "metric": METRIC, "value": world * args.steps / dev_s, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, reference factorization)",
        "config": workload_config(A, F, D.info) | {"parallelism": f"replicas x{world}"},
        "iterations": iters, "true_relres": tres,
        "e2e": {"value": world * args.steps / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n + 48},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_sweep64 (forward/backward, fp64)",
                     "bytes_per_launch": sweep_bytes, "sweep_us": sweep_s * 1e6, "peak_kind": peak_kind,
                     "iter_bytes": b_factor + b_matrix,
                     "iter_gbs": (b_factor + b_matrix) / (dev_s / args.steps / max(iters, 1)) / 1e9},
        "gpu_launches": launches_per_solve * args.steps,
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(A, F, b)
        except Exception as ex:   # the baseline is context only
            line["cpu_baseline"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    eng.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
