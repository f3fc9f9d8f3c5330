"""Solve-phase benchmark on the 3D 7-point 128^3 high-contrast SDDM grid
(n = 2,097,152): PCG solves/s and p50/p99 ms at relres 1e-8 (FP64-verified),
and the SpTRSV sweeps' HBM GB/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload grid3d_128|rmat_22|instances_256|serving_8]
                    [--k K [--lanes L] [--sweep-grid B]] [--grid G]
                    [--no-serving] [--no-serving-mix] [--no-plain] [--no-cpu-baseline]
                    [--storage fp32|fp16] [--serve-k K] [--serve-load F] [--mix-k K]

Our arm. The headline is the batched mixed-precision form: one step is one
batched PCG solve of k right-hand sides, with fp32 factor sweeps and fp64
SpMV, residual, dots and centring. k, the sweep grid and the number of lanes
are picked by the autotuner (apxchol_b200/autotune.py) unless --k is given.
The right-hand sides
come from a pool of 5 sets of N(0,1) vectors (5 is coprime with the 1-4
lanes): within a step every lane solves a different set, and a lane's set
changes from one step to the next. The line reports:
  * value      solves/s over K device-resident steps: every lane (a batch on
               its own stream, apxchol_b200/lanes.py) solves K batches back to
               back, the lanes joined once at the end; CUDA events on lane 0's
               stream, which waits for every lane.
  * e2e        the same solves through the public C ABI (apxb_batch_solve)
               from pinned host buffers: B uploaded and X downloaded inside the
               timed region.
  * plain_fp64 the plain single-RHS fp64 path (apxb_pcg; sweeps reproducing
               the reference's arithmetic), its solves/s and the speed-up.
  * serving    an open-loop Poisson request stream through SolveServer
               (continuous batching; 16 slots per lane unless --serve-k) at 70%
               of the server's own saturation throughput, measured first,
               tolerance drawn from {1e-6, 1e-8, 1e-10}: solves/s and p50/p99
               latency from arrival to result.
  * admission_ms  host time to make a new matrix solvable: factor
               preparation (on the device), the permuted operator and a k-slot
               batch with its plans; the median of three admissions (the
               "admission" field holds the samples and their breakdown).
  * serving_mix  the 8-matrix serving workload (serving_8 below) at 50, 200
               and 800 req/s: solves/s, p50/p99 and not-converged per rate,
               with two matrices admitted mid-stream under a 60 GB budget.
  * roofline   the fp32 k-RHS sweep kernel: algorithmic bytes per sweep
               (nnz_s*8 + 4(m+1) + 2*m*4*k) / measured sweep time, against the
               measured HBM copy bandwidth. iter_frac: the factor + matrix bytes
               of one PCG iteration (460 MB at 128^3) over the batch's time per
               iteration; iter_all_frac: all the iteration's algorithmic bytes
               (factor, matrix and every vector pass) over that time.
  * cpu_baseline  the reference's own cpu_solver (oracle/_ref; its x86-64-v4
               build on an AVX-512 host) on the host's physical cores: median of
               8 solves of fresh seeded right-hand sides, and its omp_sptrsv
               sweep pair. Those are the first right-hand sides lane 0 solved,
               so oracle_err_max is the largest relative error of the batched
               mixed-precision solutions against the reference's FP64 ones.
Inputs exceed L2 (factor + operator > 400 MB per iteration), so no flush is needed.

--workload selects the other configurations (one JSON line each): rmat_22 (an
R-MAT scale-22 Laplacian), instances_256 (256 uneven SDDM instances in one
batch), serving_8 (8 resident matrices under open-loop Poisson arrivals at 50,
200 and 800 requests/s, p50/p99 per rate). --grid G swaps the 128^3 grid for
G^3, a quicker check; the config's "l2" note says whether its inputs fit in L2.

--impl reference: the reference's CPU solve phase (rank 0 only) on the host's
physical cores, each step one solve of a right-hand side from a pool of 5;
prints the same JSON line with "impl": "reference".

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

METRIC = "PCG solves/s and p50/p99 ms at relres 1e-8 (FP64); SpTRSV HBM GB/s"
TOL = 1e-8
MAX_ITER = 500
FACTOR_SEED = 1
FACTOR_THREADS = 8
POOL = 5            # distinct right-hand-side sets cycled through the steps (coprime with 1-4 lanes)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def build_problem(grid_n: int):
    from apxchol_b200 import gen, refsetup
    t0 = time.time()
    A = gen.grid3d(grid_n, seed=1)
    t1 = time.time()
    F = refsetup.factorize(A, seed=FACTOR_SEED, threads=FACTOR_THREADS)
    t2 = time.time()
    log(f"[bench] grid3d_{grid_n}: n={A.n} nnz(A)={A.nnz} gen {t1 - t0:.1f}s; factor nnz={F.nnz} "
        f"rounds={len(F.rounds)} factorize {t2 - t1:.1f}s")
    return A, F


L2_BYTES = 126 * 2**20   # B200 L2


def workload_config(grid_n, A, F, form: str, extra=None):
    # bytes an iteration streams: both factor directions (4 B index + 4 B value) and the operator
    # (4 B index + 8 B value)
    it_bytes = 2 * int(F.nnz) * 8 + int(A.nnz) * 12
    l2 = (f"inputs larger than L2 (factor + operator {it_bytes / 1e6:.0f} MB per iteration), no flush"
          if it_bytes > L2_BYTES else
          f"inputs fit in L2 ({it_bytes / 1e6:.1f} MB per iteration): a small test size, not a bench workload")
    cfg = {"workload": f"grid3d_{grid_n} 7-point, weights 10^U[-3,3] (seed 1), boundary +1 (SDDM); {form}",
           "n": int(A.n), "nnz_A": int(A.nnz), "nnz_factor": int(F.nnz), "tol": TOL, "max_iter": MAX_ITER,
           "factor": f"apxchol factorize seed {FACTOR_SEED}, {FACTOR_THREADS} threads, block_greedy/vec_pool",
           "l2": l2}
    if extra:
        cfg.update(extra)
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


def profiled_traffic(k: int, grid_n: int):
    """DRAM bytes per launch of the batched sweep from the committed ncu summary
    for this k and grid (profiles/k_dw32_k{k}_grid3d_{grid}.md), else None."""
    import re
    p = os.path.join(ROOT, "profiles", f"k_dw32_k{k}_grid3d_{grid_n}.md")
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", open(p).read())
        return (int(m.group(1)), os.path.relpath(p, ROOT)) if m else (None, None)
    except OSError:
        return None, None


def max_over_ranks(values, world: int, device):
    """Element-wise max of a list of floats over all ranks (identity at world 1)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def from_rank0(values, world: int, device):
    """Rank 0's list of floats on every rank (identity at world 1)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.broadcast(t, src=0)
    return [float(v) for v in t.cpu()]


def cpu_baseline(A, F, rhs, samples: int = 8, X_gpu=None):
    """The reference cpu_solver on this host's physical cores: `samples` solves
    of fresh seeded right-hand sides rhs(0), rhs(1), ... (median time), and its
    omp_sptrsv forward + backward pair. X_gpu[c] (optional): the GPU's
    batched mixed-precision solution of rhs(c); each one's relative error
    against the reference solution of the same system is reported."""
    import oracle
    if not oracle.ref_available():
        return None
    lib = oracle.use_fastest_ref()
    cores = oracle.host_cores()
    oracle.set_threads(cores)
    R = oracle.Ref(A, F)
    times, its, tres, errs = [], [], [], []
    for j in range(samples):
        b = rhs(j)
        x, it, res, secs = R.solve(b, TOL, MAX_ITER)
        times.append(secs)
        its.append(int(it))
        tres.append(float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)))
        if X_gpu is not None and j < len(X_gpu):
            errs.append(float(np.linalg.norm(X_gpu[j] - x) / np.linalg.norm(x)))
    pair = R.pair_seconds(np.random.default_rng(5).standard_normal(R.m), 5)
    med = statistics.median(times)
    out = {"value": 1.0 / med, "unit": "solves/s", "cores": cores, "kind": "reference",
           "sample": f"{samples} solves of fresh seeded right-hand sides (median {med * 1e3:.0f} ms, "
                     f"{min(its)}-{max(its)} iterations), reference cpu_solver ({lib}) "
                     f"OMP_NUM_THREADS={cores} physical cores",
           "iterations": [min(its), max(its)], "true_relres_max": max(tres),
           "omp_sptrsv_pair_ms": pair * 1e3}
    if errs:
        out["oracle_err"] = errs
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    from apxchol_b200 import gen
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
        return 0
    A, F = build_problem(args.grid)
    pool = [gen.rhs(A.n, 1000 + j, False) for j in range(POOL)]
    lib = oracle.use_fastest_ref()
    cores = oracle.host_cores()
    oracle.set_threads(cores)
    R = oracle.Ref(A, F)
    for j in range(args.warmup):
        R.solve(pool[j % POOL], TOL, MAX_ITER)
    secs, its = [], []
    for j in range(args.steps):
        b = pool[j % POOL]           # a different right-hand side each step
        x, it, res, s = R.solve(b, TOL, MAX_ITER)
        secs.append(s)
        its.append(it)
    total = sum(secs)
    v = args.steps / total
    tres = float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": workload_config(args.grid, A, F, "reference cpu_solver, 1 RHS per solve"),
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                             "sample": f"{args.steps} solves of {POOL} cycled seeded right-hand sides, reference "
                                       f"cpu_solver ({lib}) OMP_NUM_THREADS={cores} physical cores"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "iterations": int(its[-1]), "true_relres": tres}
    print(json.dumps(line), flush=True)
    return 0


def serving_run(A, F, k, nlanes, grid, iters_per_step, load, n_req, seed, log_fn):
    """Open-loop Poisson requests through SolveServer at `load` times the
    server's own saturation throughput (measured first: 2 k lanes requests
    submitted at once, drained); returns its summary."""
    from apxchol_b200 import gen
    from apxchol_b200.serve import SolveServer, latency_stats
    srv = SolveServer(k=k, iters_per_step=iters_per_step, lanes=nlanes, sweep_grid=grid)
    try:
        srv.register("g", A, F)
        srv.admit_matrix("g")
        pool = [gen.rhs(A.n, 7000 + j, False) for j in range(8)]
        for j in range(k * nlanes):              # warm the graphs
            srv.submit("g", pool[j % 8], TOL)
        srv.drain()
        srv.completed.clear()
        t0 = time.perf_counter()
        for j in range(2 * k * nlanes):          # saturation throughput
            srv.submit("g", pool[j % 8], TOL)
        srv.drain()
        capacity = 2 * k * nlanes / (time.perf_counter() - t0)
        srv.completed.clear()
        rate = load * capacity
        rng = np.random.default_rng(seed)
        t = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
        tols = (1e-6, 1e-8, 1e-10)
        arrivals = [(float(t[j]), "g", pool[j % 8], tols[int(rng.integers(3))]) for j in range(n_req)]
        t0 = time.perf_counter()
        done = srv.run_open_loop(arrivals)
        wall = time.perf_counter() - t0
        st = latency_stats(done)
        bad = sum(1 for q in done if q.status != 0)
        # fp64 check of a sample of results against the original A
        worst = 0.0
        for q in done[:: max(1, len(done) // 16)]:
            worst = max(worst, float(np.linalg.norm(q.b - A.matvec(q.x)) / np.linalg.norm(q.b)) / q.tol)
        out = {"rate_req_s": rate, "requests": len(done), "solves_s": len(done) / wall, "p50_ms": st["p50_ms"],
               "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "capacity_solves_s": capacity, "load": load,
               "k": k, "iters_per_step": iters_per_step,
               "lanes": nlanes, "not_converged": bad, "max_true_relres_over_tol": worst}
        log_fn(f"[bench] serving {rate:.0f} req/s: {out['solves_s']:.1f} solves/s, p50 {st['p50_ms']:.1f} ms, "
               f"p99 {st['p99_ms']:.1f} ms, {bad} not converged, worst fp64 relres/tol {worst:.2f}")
        return out
    finally:
        srv.close()


def run_ours(args, rank, world, local_rank):
    import torch
    from apxchol_b200 import autotune, gen, native
    from apxchol_b200.lanes import Lanes

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    A, F = build_problem(args.grid)
    n = A.n
    eng = native.Engine(local_rank)
    t0 = time.time()
    prec = native.PREC_FP16 if args.storage == "fp16" else native.PREC_FP32
    D32 = native.DeviceFactor(eng, F, precision=prec)
    Op = native.DeviceOperator(eng, A, F.perm)
    log(f"[bench] upload {args.storage} factor + operator {time.time() - t0:.1f}s; stored nnz {D32.info.nnz_stored}; "
        f"levels {D32.info.fwd_levels}")
    stream = torch.cuda.ExternalStream(eng.stream)

    def rhs(j):
        return gen.rhs(n, 1000 + 100000 * rank + j, False)

    # ---- pick k, the sweep grid and the lane count ----
    tuned = None
    if args.k:
        k, grid, nlanes = args.k, args.sweep_grid, max(1, args.lanes)
    else:
        lg = log if rank == 0 else None
        ch = autotune.tune(eng, D32, Op, rhs, tol=TOL, max_iter=MAX_ITER, log=lg)
        k, grid, nlanes, best = ch.k, ch.grid, 1, ch.solves_per_s
        tuned = [{"k": t[0], "lanes": 1, "grid": t[1] or "resident", "solves_s": t[2]} for t in ch.table]
        for nl, g, sps, _ in autotune.tune_lanes(A, F, rhs, k, tol=TOL, max_iter=MAX_ITER, device=local_rank, log=lg,
                                                 precision=prec):
            tuned.append({"k": k, "lanes": nl, "grid": g, "solves_s": sps})
            if sps > best:
                grid, nlanes, best = g, nl, sps
    k, grid, nlanes = (int(v) for v in from_rank0([k, grid, nlanes], world, dev))   # every replica runs rank 0's choice
    D32.close()
    Op.close()
    # admission: what a new matrix costs before its first solve -- the factor
    # (prepared on the device), the permuted operator and a k-slot batch. Three
    # admissions, the median reported; objects left by the tuning are collected
    # first, so that no destructor's device free lands inside a timed admission.
    import gc
    gc.collect()
    adm = []
    for _ in range(3):
        torch.cuda.synchronize()
        t_adm = time.perf_counter()
        Da = native.DeviceFactor(eng, F, precision=prec)
        t_f = time.perf_counter()
        Oa = native.DeviceOperator(eng, A, F.perm)
        t_o = time.perf_counter()
        Ba = native.Batch(eng, [Da], [Oa], k)
        eng.sync()
        t_b = time.perf_counter()
        Ba.close(); Oa.close(); Da.close()
        adm.append([(t_b - t_adm) * 1e3, (t_f - t_adm) * 1e3, (t_o - t_f) * 1e3, (t_b - t_o) * 1e3])
    admission_ms = float(np.median([a[0] for a in adm]))
    admission = {"median_ms": admission_ms, "samples_ms": [round(a[0], 1) for a in adm],
                 "factor_ms": [round(a[1], 1) for a in adm], "operator_ms": [round(a[2], 1) for a in adm],
                 "batch_ms": [round(a[3], 1) for a in adm], "k": k}
    log(f"[bench] admission (factor + operator + k={k} batch), 3 times: " +
        ", ".join(f"{a[0]:.0f} ms ({a[1]:.0f} + {a[2]:.0f} + {a[3]:.0f})" for a in adm))
    lanes = Lanes(A, F, k, lanes=nlanes, grid=grid, device=local_rank, precision=prec)
    grid = lanes.grid
    bt = lanes.lanes[0].batch
    streams = [torch.cuda.ExternalStream(h) for h in lanes.streams]
    sets = []
    for p in range(POOL):
        Bf, nrhs = lanes.pack(np.stack([rhs(p * k + c) for c in range(k)]))
        sets.append((Bf, torch.from_numpy(Bf).to(dev)))
    dXs = [torch.empty_like(sets[0][1]) for _ in range(nlanes)]
    torch.cuda.synchronize()

    def step_dev(i, flags=native.DEVICE_PTRS):
        # lane j solves set (i * lanes + j) of the pool
        return lanes.solve_raw([sets[(i * nlanes + j) % POOL][1] for j in range(nlanes)], dXs, nrhs, tol=TOL,
                               max_iter=MAX_ITER, flags=flags)

    for i in range(args.warmup):
        step_dev(i)
    # FP64 verification of every slot of one step, on the device and on the host
    res = step_dev(0, native.DEVICE_PTRS | native.TRUE_RESIDUAL)
    its = [r.iterations for lane in res for r in lane[:k]]
    dev_tres = max(r.true_residual for lane in res for r in lane[:k])
    host_tres = 0.0
    x_lane0 = None   # lane 0 solved set 0: right-hand sides rhs(0) .. rhs(k - 1)
    for j in range(nlanes):
        X0, B0 = dXs[j].cpu().numpy(), sets[j % POOL][0]
        if j == 0:
            x_lane0 = [X0[c * n:(c + 1) * n].copy() for c in range(k)]
        for c in range(k):
            bcol, xcol = B0[c * n:(c + 1) * n], X0[c * n:(c + 1) * n]
            host_tres = max(host_tres, float(np.linalg.norm(bcol - A.matvec(xcol)) / np.linalg.norm(bcol)))
    log(f"[bench] rank {rank}: k={k} lanes={nlanes} grid={grid or 'resident'}: iterations {min(its)}-{max(its)}, "
        f"fp64 true relres max {host_tres:.2e} (device {dev_tres:.2e})")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- value: device-resident batched solves ----
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lane_ev = [torch.cuda.Event() for _ in streams]

    def open_region():
        # every lane's stream starts after ev0 on lane 0's stream
        ev0.record(streams[0])
        for st in streams[1:]:
            st.wait_event(ev0)

    def close_region():
        # ev1 on lane 0's stream after every lane's work
        for st, e in zip(streams, lane_ev):
            e.record(st)
            streams[0].wait_event(e)
        ev1.record(streams[0])

    def lane_steps(flags, bufs, outs):
        # each lane solves its `steps` batches back to back (lane j, step i: set (i * lanes + j));
        # the lanes are joined once, at the end of the timed region
        def run(j, lane):
            its = []
            for i in range(args.steps):
                r = lane.batch.solve_raw(bufs[((i + 1) * nlanes + j) % POOL], outs[j], nrhs, tol=TOL,
                                         max_iter=MAX_ITER, flags=flags)
                its.append(max(x.iterations for x in r[:k]))
            return its
        return lanes.each(run)

    dev_bufs = [s_[1] for s_ in sets]
    with ClockSampler(local_rank) as clk:
        barrier()
        open_region()
        per_lane = lane_steps(native.DEVICE_PTRS, dev_bufs, dXs)
        close_region()
        barrier()
    dev_s = ev0.elapsed_time(ev1) * 1e-3
    iters_timed = [max(col) for col in zip(*per_lane)]
    # ---- e2e: pinned host buffers through the C ABI (apxb_batch_solve, one call per lane) ----
    hB = [torch.from_numpy(s[0]).pin_memory() for s in sets]
    hX = [torch.empty(n * k, dtype=torch.float64).pin_memory() for _ in range(nlanes)]

    def step_host(i):
        return lanes.solve_raw([hB[(i * nlanes + j) % POOL] for j in range(nlanes)], hX, nrhs, tol=TOL,
                               max_iter=MAX_ITER, flags=0)

    step_host(0)
    barrier()
    open_region()
    lane_steps(0, hB, hX)
    close_region()
    barrier()
    e2e_s = ev0.elapsed_time(ev1) * 1e-3
    # ---- roofline: the batches' own fp32 k-RHS sweeps, all lanes running them at once ----
    st = lanes.sweep_timed(10)
    fwd_s = sum(t[0] for t in st) / len(st)
    bck_s = sum(t[1] for t in st) / len(st)
    m, nnz_s = D32.info.m, D32.info.nnz_stored
    # per stored entry: index + value (fp32 4 B, fp16 2 B); fp16 adds the per-row fp32 diagonal and,
    # in the backward sweep, the fp64 inverse scale squared (4 B per row on average over the pair)
    e_bytes, r_bytes = (6, 8) if args.storage == "fp16" else (8, 0)
    sweep_bytes = nnz_s * e_bytes + 4 * (m + 1) + r_bytes * m + 2 * m * 4 * k
    sweep_s = (fwd_s + bck_s) / 2
    peak, peak_kind = measured_peak_hbm()
    achieved = sum(2 * sweep_bytes / (t[0] + t[1]) for t in st) / 1e9   # summed over the concurrent lanes
    traffic, traffic_src = profiled_traffic(k, args.grid)
    b_iter = 2 * (nnz_s * e_bytes + 4 * (m + 1) + r_bytes * m) + A.nnz * 12 + 4 * (n + 1)
    b_iter *= nlanes   # every lane reads the factor and the matrix once per iteration
    iter_s = dev_s / max(1, sum(iters_timed))
    iter_gbs = b_iter / iter_s / 1e9
    # all algorithmic traffic of one batched iteration (every vector pass the kernels make), per lane:
    # SpMV (A, p gathered once, Ap written), r update (r, Ap read; r and the fp32 sweep input
    # written), two sweeps (factor, input read, output and re-armed buffer written), r.z (r, z read),
    # x and p update (x, p, z read; x, p written)
    v8, v4 = 8 * n * k, 4 * n * k
    b_all = (A.nnz * 12 + 4 * (n + 1) + 2 * v8) + (3 * v8 + v4) + \
        2 * (nnz_s * e_bytes + 4 * (m + 1) + r_bytes * m + 3 * v4) + (v8 + v4) + (v4 + 4 * v8)
    b_all *= nlanes
    iter_all_gbs = b_all / iter_s / 1e9
    dev_s, e2e_s = max_over_ranks([dev_s, e2e_s], world, dev)
    lanes.close()

    # ---- plain fp64 single-RHS path ----
    plain = None
    if not args.no_plain:
        # context beside the headline: a failure here is reported in its field, not fatal
        try:
            D64 = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
            Op = native.DeviceOperator(eng, A, F.perm)
            db = torch.from_numpy(rhs(0)).to(dev)
            dx = torch.empty_like(db)
            for _ in range(3):
                native.pcg(eng, D64, Op, db, dx, tol=TOL, max_iter=MAX_ITER, device_ptrs=True, true_residual=False)
            ns = max(3, min(args.steps, 8))
            secs, pits = [], 0
            for j in range(ns):
                _, r = native.pcg(eng, D64, Op, sets[j % POOL][1][:n], dx, tol=TOL, max_iter=MAX_ITER, device_ptrs=True,
                                  true_residual=False)
                secs.append(r.seconds)
                pits = r.iterations
            dm = torch.from_numpy(np.random.default_rng(5).standard_normal(m)).to(dev)
            dz = torch.empty_like(dm)
            D64.sweep_pair_timed(dm, dz, 3)
            pair64 = D64.sweep_pair_timed(dm, dz, 10)
            b64 = nnz_s * 8 + 4 * (m + 1) + 2 * m * 8
            plain = {"solves_s": ns / sum(secs), "ms_per_solve": sum(secs) / ns * 1e3, "iterations": pits,
                     "sweep_us": pair64 / 2 * 1e6, "sweep_gbs": b64 / (pair64 / 2) / 1e9}
            D64.close()
            Op.close()
            log(f"[bench] plain fp64: {plain['solves_s']:.1f} solves/s ({plain['ms_per_solve']:.1f} ms, {pits} it), "
                f"fp64 sweep {plain['sweep_us']:.0f} us = {plain['sweep_gbs']:.0f} GB/s")
        except Exception as ex:
            plain = {"error": f"{type(ex).__name__}: {ex}"}
            log(f"[bench] plain fp64 failed: {ex}")

    value = world * args.steps * k * nlanes / dev_s
    mix = None
    if not args.no_serving_mix and rank == 0:
        try:   # the 8-matrix serving workload beside the headline (reported in its field)
            rates, resident_gb = serving_mix(local_rank, k=args.mix_k)
            mix = {"workload": "serving_8: 8 matrices (2 x 2D grid 1024^2, 2 x 3D grid 96^3, 2 x R-MAT scale 20 "
                               f"LCC, 2 x random 6-regular n=500k), Poisson arrivals, 60 GB budget, k={args.mix_k}",
                   "rates": rates, "resident_gb": resident_gb}
        except Exception as ex:
            mix = {"error": f"{type(ex).__name__}: {ex}"}
            log(f"[bench] serving mix failed: {ex}")
    serving = None
    if not args.no_serving and rank == 0:
        try:
            sk = min(k, args.serve_k)
            serving = serving_run(A, F, sk, nlanes, grid, args.iters_per_step, args.serve_load,
                                  args.serve_requests, 11, log)
        except Exception as ex:   # reported in its field; the headline stands
            serving = {"error": f"{type(ex).__name__}: {ex}"}
            log(f"[bench] serving failed: {ex}")

    if rank != 0:
        eng.close()
        return 0
    mean_its = sum(iters_timed) / max(1, len(iters_timed))
    # per batched solve: admit; per iteration 12 kernels plus the residual refresh's SpMV, update and
    # verification finalize (on by default; no long rows here); x out
    launches_per_step = nlanes * (1 + 15 * (mean_its + 1) + 3)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 sweeps / f64 outer" + (" (fp16 factor storage)" if args.storage == "fp16" else ""),
        "data": "synthetic (seeded generator, reference factorization)",
        "config": workload_config(args.grid, A, F, f"batched mixed precision, {nlanes} lane(s) x {k} RHS per step",
                                  {"k": k, "lanes": nlanes, "sweep_grid": grid or "resident", "rhs_sets": POOL,
                                   "factor_storage": args.storage, "parallelism": f"replicas x{world}"}),
        "iterations": [min(iters_timed), max(iters_timed)], "true_relres_max": host_tres,
        "e2e": {"value": world * args.steps * k * nlanes / e2e_s, "unit": "solves/s",
                "h2d_bytes_per_step": 8 * n * k * nlanes, "d2h_bytes_per_step": (8 * n * k + 24 * k) * nlanes},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_source": traffic_src,
                     "kernel": f"k_dw32<DIR,{k},{'true' if args.storage == 'fp16' else 'false'}> (batched fp32 "
                               f"sweep, {args.storage} factor storage, {k} RHS, {nlanes} concurrent lane(s), "
                               f"{grid or 'resident'} blocks each)",
                     "bytes_per_launch": sweep_bytes, "fwd_us": fwd_s * 1e6, "bck_us": bck_s * 1e6,
                     "peak_kind": peak_kind, "iter_bytes": b_iter, "iter_gbs": iter_gbs, "iter_frac": iter_gbs / peak,
                     "iter_all_bytes": b_all, "iter_all_gbs": iter_all_gbs, "iter_all_frac": iter_all_gbs / peak},
        "plain_fp64": plain,
        "speedup_vs_plain_fp64": (value / world) / plain["solves_s"] if plain and "solves_s" in plain else None,
        "serving": serving,
        "serving_mix": mix,
        "admission_ms": admission_ms,
        "admission": admission,
        "autotune": tuned,
        "gpu_launches": int(round(launches_per_step * args.steps)),
        "clocks": clk.summary(),
    }
    if not args.no_cpu_baseline:
        try:
            # the reference solves the first right-hand sides lane 0 solved, so the batched mixed-precision
            # solutions get their error against the FP64 reference solution of the same systems
            cb = cpu_baseline(A, F, rhs, X_gpu=x_lane0)
            line["cpu_baseline"] = cb
            if cb and cb.get("oracle_err"):
                line["oracle_err_max"] = max(cb["oracle_err"])
                line["oracle_err_note"] = (f"max over {len(cb['oracle_err'])} batched mixed-precision solutions of "
                                           "||x - x_ref|| / ||x_ref||, x_ref the reference cpu_solver's FP64 "
                                           "solution of the same system at the same tolerance")
        except Exception as ex:   # the baseline is context only
            line["cpu_baseline"] = {"error": str(ex)}
    print(json.dumps(line), flush=True)
    eng.close()
    return 0


def _verify(A, B_rows, X_rows):
    """Largest FP64 relative residual ||b - A x|| / ||b|| over the given columns."""
    worst = 0.0
    for b, x in zip(B_rows, X_rows):
        worst = max(worst, float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)))
    return worst


def run_rmat22(args, rank, world, local_rank):
    """R-MAT scale-22 Laplacian: batched mixed precision (autotuned k), the plain
    FP64 path, and one reference cpu_solver solve (iterations, time)."""
    import torch
    import oracle
    from apxchol_b200 import autotune, gen, native, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    A, F = workloads.rmat_22(log)
    n = A.n
    rhs = lambda j: gen.rhs(n, 3000 + j, True)
    eng = native.Engine(local_rank)
    D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    Op = native.DeviceOperator(eng, A, F.perm)
    ch = autotune.tune(eng, D32, Op, rhs, tol=TOL, max_iter=MAX_ITER, ks=(1, 4, 8, 16, 32, 64, 128), grids=(0,), log=log)
    k = ch.k
    bt = native.Batch(eng, [D32], [Op], k)
    B = np.stack([rhs(c) for c in range(k)])
    Bf, nrhs = bt.pack([B])
    dB = torch.from_numpy(Bf).to(dev)
    dX = torch.empty_like(dB)
    stream = torch.cuda.ExternalStream(eng.stream)
    for _ in range(args.warmup):
        bt.solve_raw(dB, dX, nrhs, tol=TOL, max_iter=MAX_ITER, flags=native.DEVICE_PTRS)
    steps = max(1, min(args.steps, 5))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        res = bt.solve_raw(dB, dX, nrhs, tol=TOL, max_iter=MAX_ITER, flags=native.DEVICE_PTRS)
    ev1.record(stream)
    torch.cuda.synchronize()
    secs = ev0.elapsed_time(ev1) * 1e-3
    X = dX.cpu().numpy()
    tres = _verify(A, [B[c] for c in range(k)], [X[c * n:(c + 1) * n] for c in range(k)])
    its = [res[c].iterations for c in range(k)]
    bt.close(); D32.close()
    D64 = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    x64, r64 = native.pcg(eng, D64, Op, B[0], tol=TOL, max_iter=MAX_ITER)
    _, r64 = native.pcg(eng, D64, Op, B[0], tol=TOL, max_iter=MAX_ITER)
    tres64 = _verify(A, [B[0]], [x64])
    D64.close(); Op.close(); eng.close()
    ref = None
    if oracle.ref_available():
        lib = oracle.use_fastest_ref()
        cores = oracle.host_cores()
        oracle.set_threads(cores)
        xr, itr, _, sr = oracle.Ref(A, F).solve(B[0], TOL, MAX_ITER)
        xa, xb = X[:n] - X[:n].mean(), xr - xr.mean()   # a Laplacian's solutions, compared up to the null space
        err = float(np.linalg.norm(xa - xb) / np.linalg.norm(xb))   # batched slot 0 against the reference
        ref = {"iterations": int(itr), "seconds": sr, "solves_s": 1.0 / sr, "cores": cores, "lib": lib,
               "oracle_err_slot0": err}
    line = {"metric": METRIC, "value": k * steps / secs, "unit": "solves/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": secs / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 sweeps / f64 outer", "data": "synthetic (seeded generator)",
            "config": {"workload": "rmat_22 LCC Laplacian, batched mixed precision", "n": n, "nnz_A": int(A.nnz),
                       "nnz_factor": int(F.nnz), "k": k, "tol": TOL},
            "iterations": [min(its), max(its)], "true_relres_max": tres,
            "plain_fp64": {"solves_s": 1.0 / r64.seconds, "iterations": r64.iterations, "true_relres": tres64},
            "reference_cpu": ref,
            "autotune": [{"k": t[0], "solves_s": t[2]} for t in ch.table]}
    print(json.dumps(line), flush=True)
    return 0


def run_instances256(args, rank, world, local_rank):
    """256 uneven SDDM instances in one batch (autotuned k)."""
    import torch
    from apxchol_b200 import autotune, gen, native, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    insts = workloads.instances_256(log)
    eng = native.Engine(local_rank)
    Ds = [native.DeviceFactor(eng, F, precision=native.PREC_FP32) for _, F, _ in insts]
    Ops = [native.DeviceOperator(eng, A, F.perm) for A, F, _ in insts]
    rhs = [np.stack([gen.rhs(A.n, 5000 + 10 * i + j, False) for j in range(c)]) for i, (A, F, c) in enumerate(insts)]
    total = sum(r.shape[0] for r in rhs)
    k, table = autotune.tune_instances(eng, Ds, Ops, rhs, tol=TOL, max_iter=MAX_ITER, log=log)
    bt = native.Batch(eng, Ds, Ops, k)
    cmax = max(r.shape[0] for r in rhs)
    passes = []
    for p0 in range(0, cmax, k):
        part = [r[p0:p0 + k] if r.shape[0] > p0 else np.zeros((0, r.shape[1])) for r in rhs]
        Bf, nrhs = bt.pack(part)
        passes.append((torch.from_numpy(Bf).to(dev), nrhs, part))
    dX = torch.empty_like(passes[0][0])
    stream = torch.cuda.ExternalStream(eng.stream)
    for _ in range(args.warmup):
        for dB, nrhs, _ in passes:
            bt.solve_raw(dB, dX, nrhs, tol=TOL, max_iter=MAX_ITER, flags=native.DEVICE_PTRS)
    steps = max(1, min(args.steps, 5))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        for dB, nrhs, _ in passes:
            bt.solve_raw(dB, dX, nrhs, tol=TOL, max_iter=MAX_ITER, flags=native.DEVICE_PTRS)
    ev1.record(stream)
    torch.cuda.synchronize()
    secs = ev0.elapsed_time(ev1) * 1e-3
    worst, bad = 0.0, 0
    for dB, nrhs, part in passes:
        res = bt.solve_raw(dB, dX, nrhs, tol=TOL, max_iter=MAX_ITER, flags=native.DEVICE_PTRS | native.TRUE_RESIDUAL)
        for i, q in enumerate(part):
            for c in range(q.shape[0]):
                r = res[i * k + c]
                worst = max(worst, r.true_residual)
                bad += r.status != 0
    line = {"metric": METRIC, "value": total * steps / secs, "unit": "solves/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": secs / steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 sweeps / f64 outer", "data": "synthetic (seeded generator)",
            "config": {"workload": "instances_256: uneven SDDM instances in one batch", "instances": len(insts),
                       "sum_n": int(sum(A.n for A, _, _ in insts)), "rhs": total, "k": k, "passes": len(passes),
                       "tol": TOL},
            "true_relres_max": worst, "not_converged": int(bad),
            "autotune": [{"k": t[0], "solves_s": t[1]} for t in table]}
    bt.close()
    for o in Ops + Ds:
        o.close()
    eng.close()
    print(json.dumps(line), flush=True)
    return 0


def serving_mix(device, sweep_grid=None, log_fn=log, k: int = 8):
    """The 8-matrix serving workload (C5): 8 registered matrices, 6 resident at
    the start, open-loop Poisson requests at 50 / 200 / 800 req/s (matrix
    uniform, tolerance from {1e-6, 1e-8, 1e-10}, >= 1000 requests per rate);
    the two matrices not resident are admitted when their first request
    arrives, under a 60 GB budget; k slots per resident matrix. Returns (rates, resident GB)."""
    from apxchol_b200 import gen, workloads
    from apxchol_b200.serve import SolveServer, latency_stats
    mats = workloads.serving_8(log_fn)
    srv = SolveServer(device=device, budget_bytes=60 * 10**9, k=k, iters_per_step=2, sweep_grid=sweep_grid or None)
    rates = []
    try:
        for name, A, F in mats:
            srv.register(name, A, F)
        for name, A, F in mats[:6]:
            srv.admit_matrix(name)
            for j in range(8):
                srv.submit(name, gen.rhs(A.n, 10 + j, not F.sddm), TOL)
        srv.drain()
        srv.completed.clear()
        pools = {name: [gen.rhs(A.n, 100 + j, not F.sddm) for j in range(4)] for name, A, F in mats}
        names = [nm for nm, _, _ in mats]
        for rate, nreq in ((50, 1000), (200, 1000), (800, 2400)):   # p50/p99 over >= 1000 requests per rate
            rng = np.random.default_rng(rate)
            t = np.cumsum(rng.exponential(1.0 / rate, size=nreq))
            tols = (1e-6, 1e-8, 1e-10)
            arrivals = [(float(t[j]), names[int(rng.integers(len(names)))], None, tols[int(rng.integers(3))])
                        for j in range(nreq)]
            arrivals = [(dt, nm, pools[nm][j % 4], tol) for j, (dt, nm, _, tol) in enumerate(arrivals)]
            adm0 = srv.admissions
            t0 = time.perf_counter()
            done = srv.run_open_loop(arrivals)
            wall = time.perf_counter() - t0
            st = latency_stats(done)
            rates.append({"rate_req_s": rate, "requests": len(done), "solves_s": len(done) / wall,
                          "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "not_converged": sum(q.status != 0 for q in done),
                          "matrix_admissions": srv.admissions - adm0})
            log_fn(f"[bench] serving_8 {rate} req/s: {len(done) / wall:.1f} solves/s, p50 {st['p50_ms']:.1f} ms, "
                   f"p99 {st['p99_ms']:.1f} ms")
        resident_gb = srv.used_bytes() / 1e9
    finally:
        srv.close()
    return rates, resident_gb


def run_serving8(args, rank, world, local_rank):
    """8 resident matrices, open-loop Poisson requests at 50/200/800 req/s
    (matrix uniform, tol from {1e-6, 1e-8, 1e-10}); two matrices are admitted
    only when their first request arrives (60 GB budget)."""
    import torch
    torch.cuda.set_device(local_rank)
    rates, resident_gb = serving_mix(local_rank, args.sweep_grid, k=args.mix_k)
    line = {"metric": METRIC, "value": rates[-1]["solves_s"], "unit": "solves/s", "n_gpus": world, "steps": len(rates),
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 sweeps / f64 outer", "data": "synthetic (seeded generator)",
            "config": {"workload": "serving_8: 8 matrices, Poisson arrivals", "k": args.mix_k, "budget_gb": 60,
                       "sweep_grid": args.sweep_grid or "auto (resident grid / 4)",
                       "resident_gb": resident_gb},
            "serving": rates}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=128, help="grid side (the workload is 128)")
    ap.add_argument("--k", type=int, default=0, help="right-hand sides per step (0 = autotune)")
    ap.add_argument("--sweep-grid", type=int, default=0, help="sweep blocks per lane with --k (0 = resident / lanes)")
    ap.add_argument("--lanes", type=int, default=1, help="concurrent batches (streams) with --k")
    ap.add_argument("--iters-per-step", type=int, default=2, help="serving: iterations per server step")
    ap.add_argument("--serve-requests", type=int, default=1000)
    ap.add_argument("--mix-k", type=int, default=8, help="serving mix: slots per resident matrix")
    ap.add_argument("--storage", choices=["fp32", "fp16"], default="fp32",
                    help="batched factor storage: fp32 values, or the reference GPU default fp16 (column-scaled)")
    ap.add_argument("--serve-k", type=int, default=16,
                    help="serving: slots per lane (at most the batch k; fewer slots, shorter iterations, lower latency)")
    ap.add_argument("--serve-load", type=float, default=0.7,
                    help="serving: Poisson rate as a fraction of the server's measured saturation throughput")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-serving-mix", action="store_true", help="skip the 8-matrix serving field")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="grid3d_128", choices=["grid3d_128", "rmat_22", "instances_256", "serving_8"],
                    help="grid3d_128 is the benchmark; the others measure the other workloads, one JSON line each")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload != "grid3d_128":
        fn = {"rmat_22": run_rmat22, "instances_256": run_instances256, "serving_8": run_serving8}[args.workload]
        return fn(args, rank, world, local_rank)
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
