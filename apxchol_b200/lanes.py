"""Batch lanes: several k-slot batches of one matrix, each on its own engine
(CUDA stream) of one GPU, solved concurrently.

The batched sweeps are bound by the latency of the level chain: they keep
DRAM at 17-27% and leave issue slots idle. A second batch on another stream
runs its bandwidth-bound vector passes and SpMV in those gaps. Each lane's
persistent sweep grid is cut to its share of the SMs, so the lanes' sweeps
are co-resident. Lanes never wait on one another (every sweep claims its
work in level order from its own counter), so any grid is safe.

Each lane holds its own copy of the factor (fp32, or fp16 storage with
precision=native.PREC_FP16) and the operator. One lane of 128^3 at k = 16 is
about 2.6 GB of device memory.
"""
from __future__ import annotations

import threading

import numpy as np

from . import native


class Lane:
    def __init__(self, mat, fac, k: int, grid: int, device: int, precision: int = native.PREC_FP32):
        self.batch = self.op = self.factor = None
        self.eng = native.Engine(device)
        self.eng.set_sweep_grid(grid)
        try:
            self.factor = native.DeviceFactor(self.eng, fac, precision=precision)
            self.op = native.DeviceOperator(self.eng, mat, fac.perm)
            self.batch = native.Batch(self.eng, [self.factor], [self.op], k)
        except Exception:
            self.close()          # what was made so far, the engine included
            raise
        self.eng.set_sweep_grid(0)

    def close(self):
        for o in ("batch", "op", "factor", "eng"):
            if getattr(self, o, None) is not None:
                getattr(self, o).close()
                setattr(self, o, None)


class Lanes:
    """`lanes` batches of k slots over one matrix. grid: sweep blocks per lane
    (0 = the resident grid divided among the lanes); precision: the factor
    storage (native.PREC_FP32, or native.PREC_FP16)."""

    def __init__(self, mat, fac, k: int, lanes: int = 1, grid: int = 0, device: int = 0,
                 precision: int = native.PREC_FP32):
        import torch
        self.k, self.n, self.device = k, mat.n, device
        if grid <= 0 and lanes > 1:
            sms = torch.cuda.get_device_properties(device).multi_processor_count
            grid = max(1, (2 * sms) // lanes)
        self.grid = grid
        self.lanes = []
        try:
            for _ in range(lanes):
                self.lanes.append(Lane(mat, fac, k, grid, device, precision))
        except Exception:
            self.close()
            raise

    @property
    def streams(self):
        return [ln.eng.stream for ln in self.lanes]

    def pack(self, B):
        """(k, n) right-hand sides -> the flat caller layout of one lane."""
        return self.lanes[0].batch.pack([B])

    def solve_raw(self, Bs, Xs, nrhs, tol: float = 1e-8, max_iter: int = 500, flags: int = 0):
        """One batched solve per lane, concurrently: Bs[i] / Xs[i] are lane i's
        caller-layout buffers (device with native.DEVICE_PTRS, else pinned host).
        Returns each lane's per-slot results."""
        out = [None] * len(self.lanes)
        errs = []

        def run(i):
            try:
                out[i] = self.lanes[i].batch.solve_raw(Bs[i], Xs[i], nrhs, tol=tol, max_iter=max_iter, flags=flags)
            except Exception as ex:   # re-raised on the calling thread
                errs.append(ex)

        if len(self.lanes) == 1:
            run(0)
        else:
            threads = [threading.Thread(target=run, args=(i,)) for i in range(len(self.lanes))]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
        if errs:
            raise errs[0]
        return out

    def each(self, fn):
        """Run fn(i, lane) for every lane concurrently (one host thread per lane,
        joined once at the end); returns the results in lane order."""
        out = [None] * len(self.lanes)
        errs = []

        def run(i):
            try:
                out[i] = fn(i, self.lanes[i])
            except Exception as ex:   # re-raised on the calling thread
                errs.append(ex)

        threads = [threading.Thread(target=run, args=(i,)) for i in range(len(self.lanes))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errs:
            raise errs[0]
        return out

    def sweep_timed(self, reps: int = 10):
        """Every lane's forward and backward sweeps timed (CUDA events on its own
        stream) while all lanes run them concurrently: [(fwd s, bck s)] per lane."""
        return self.each(lambda i, ln: ln.batch.sweep_timed(reps))

    def memory_used(self) -> int:
        return sum(ln.eng.memory_used() for ln in self.lanes)

    def close(self):
        for ln in self.lanes:
            ln.close()
        self.lanes = []

    def __del__(self):
        self.close()


def rhs_block(rhs, k: int, first: int) -> np.ndarray:
    return np.stack([rhs(first + c) for c in range(k)])
