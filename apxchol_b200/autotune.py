"""Autotuner of the batched mixed-precision form.

For one matrix it times a whole batched solve (CUDA events, device-resident
right-hand sides) for every right-hand-side block width k in
{1, 2, 4, 8, 16, 32, 64, 128} and every candidate sweep grid (the resident grid and one block per SM), and
keeps the fastest solves/s. The sweeps' other knobs are fixed by the plan: the
lanes per row follow the row length (1, 4, 8, 16 or 32), and the in-flight
depth is the 3-stage item pipeline with 8 entries per lane, plus an L2
prefetch of the next item's dependency rows.

The reference has no autotuner; its GPU path solves one right-hand side at a
time (cuda_pcg::solve, include/apxchol/solver/pcg_cuda.h:157-261).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import native

KS = (1, 2, 4, 8, 16, 32, 64, 128)
KS_INSTANCES = (1, 2, 4, 8, 16)   # many small instances with 1-8 right-hand sides each


@dataclass
class Choice:
    k: int
    grid: int                     # 0 = the resident grid
    solves_per_s: float
    seconds_per_batch: float
    iterations: int
    table: list = field(default_factory=list)   # (k, grid, solves/s, iterations) of every candidate


def _num_sms(device: int) -> int:
    import torch
    return torch.cuda.get_device_properties(device).multi_processor_count


def time_batch(eng: native.Engine, bt: native.Batch, rhs, tol: float, max_iter: int, reps: int = 1):
    """Device seconds of one batched solve of bt.k right-hand sides (rhs(j) -> array), best of reps."""
    import torch
    B = np.stack([rhs(j) for j in range(bt.k)])
    Bf, nrhs = bt.pack([B])
    dB = torch.from_numpy(Bf).cuda(eng.device)
    dX = torch.empty_like(dB)
    res = bt.solve_raw(dB, dX, nrhs, tol=tol, max_iter=max_iter, flags=native.DEVICE_PTRS)   # warm-up
    best = float("inf")
    for _ in range(reps):
        res = bt.solve_raw(dB, dX, nrhs, tol=tol, max_iter=max_iter, flags=native.DEVICE_PTRS)
        best = min(best, res[0].seconds)
    its = max(res[c].iterations for c in range(bt.k))
    return best, its


def tune(eng: native.Engine, factor: native.DeviceFactor, op: native.DeviceOperator, rhs, tol: float = 1e-8,
         max_iter: int = 500, ks=KS, grids=None, reps: int = 1, log=None) -> Choice:
    """Pick k and the sweep grid for one matrix. rhs(j) gives the j-th right-hand side."""
    if grids is None:
        grids = (0, _num_sms(eng.device))
    table = []
    best = None
    try:
        for grid in grids:
            eng.set_sweep_grid(grid)
            for k in ks:
                bt = native.Batch(eng, [factor], [op], k)
                try:
                    secs, its = time_batch(eng, bt, rhs, tol, max_iter, reps)
                finally:
                    bt.close()
                sps = k / secs
                table.append((k, grid, sps, its))
                if log:
                    log(f"[autotune] k={k:2d} grid={grid or 'resident'}: {secs * 1e3:8.2f} ms/batch, "
                        f"{sps:8.1f} solves/s, {its} iterations")
                if best is None or sps > best.solves_per_s:
                    best = Choice(k=k, grid=grid, solves_per_s=sps, seconds_per_batch=secs, iterations=its)
    finally:
        eng.set_sweep_grid(0)
    best.table = table
    return best


def tune_lanes(mat, fac, rhs, k: int, lanes_list=(2, 3, 4), tol: float = 1e-8, max_iter: int = 500,
               device: int = 0, log=None, precision: int = native.PREC_FP32):
    """Solves/s of `lanes` concurrent k-slot batches (apxchol_b200.lanes), for
    each lane count; returns [(lanes, grid, solves/s, iterations)]."""
    import time
    import torch
    from .lanes import Lanes
    table = []
    for nl in lanes_list:
        ln = Lanes(mat, fac, k, lanes=nl, device=device, precision=precision)
        try:
            B, nrhs = ln.pack(np.stack([rhs(c) for c in range(k)]))
            dB = [torch.from_numpy(B).cuda(device) for _ in range(nl)]
            dX = [torch.empty_like(b) for b in dB]
            res = ln.solve_raw(dB, dX, nrhs, tol=tol, max_iter=max_iter, flags=native.DEVICE_PTRS)   # warm-up
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            res = ln.solve_raw(dB, dX, nrhs, tol=tol, max_iter=max_iter, flags=native.DEVICE_PTRS)
            torch.cuda.synchronize(device)
            dt = time.perf_counter() - t0
            its = max(r.iterations for lane in res for r in lane[:k])
            table.append((nl, ln.grid, nl * k / dt, its))
            if log:
                log(f"[autotune] lanes={nl} k={k} grid={ln.grid}: {dt * 1e3:8.2f} ms per round, "
                    f"{nl * k / dt:8.1f} solves/s")
        finally:
            ln.close()
            del ln
    return table


def tune_instances(eng: native.Engine, factors, ops, rhs, tol: float = 1e-8, max_iter: int = 500, ks=KS_INSTANCES,
                   log=None):
    """Pick k for a multi-instance batch: rhs[i] is instance i's (c_i, n_i)
    right-hand sides. A width k solves them in ceil(max c_i / k) passes of one
    batch; every pass is timed (device events), and the k with the highest
    total solves/s wins. Returns (k, [(k, solves/s, seconds)])."""
    total = sum(int(np.atleast_2d(b).shape[0]) for b in rhs)
    table = []
    for k in ks:
        bt = native.Batch(eng, factors, ops, k)
        try:
            cmax = max(int(np.atleast_2d(b).shape[0]) for b in rhs)
            secs = 0.0
            for p0 in range(0, cmax, k):
                part = [np.atleast_2d(b)[p0:p0 + k] for b in rhs]
                part = [q if q.shape[0] else np.zeros((0, f.n)) for q, f in zip(part, factors)]
                B, nrhs = bt.pack(part)
                X = np.empty_like(B)
                res = bt.solve_raw(B, X, nrhs, tol=tol, max_iter=max_iter)
                secs += res[0].seconds
        finally:
            bt.close()
        table.append((k, total / secs, secs))
        if log:
            log(f"[autotune] instances={len(factors)} k={k:2d}: {secs * 1e3:8.2f} ms, {total / secs:8.1f} solves/s")
    best = max(table, key=lambda t: t[1])
    return best[0], table
