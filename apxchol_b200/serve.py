"""Solve server: resident factors, continuous batching, an HBM byte budget.

Each resident matrix gets its own engine (CUDA stream), factor, operator and
a batch of k right-hand-side slots (fp32 preconditioner sweeps, fp64 PCG;
native.Batch). Requests (matrix id, right-hand side, tolerance) are admitted
into free slots at iteration boundaries while the other slots keep
iterating, and leave the moment they converge, so work of requests that
arrive while others are running overlaps on the device -- across slots of one
matrix and, through the per-matrix streams, across matrices.

Matrices are admitted against a device-memory budget; when a new matrix does
not fit, idle resident matrices are evicted least-recently-used first, and a
matrix that still does not fit is refused (BudgetError).

The reference has no serving layer; the per-request semantics are those of
its cpu_solver::solve (src/solve.cpp:478-654) with the request's tolerance.
"""
from __future__ import annotations

import collections
import concurrent.futures
import time
from dataclasses import dataclass, field

import numpy as np

from . import native


class BudgetError(RuntimeError):
    pass


@dataclass
class Request:
    rid: int
    mid: object
    b: np.ndarray
    tol: float
    arrival: float                 # host clock (time.perf_counter) when it was submitted
    start: float = 0.0             # when it entered a slot
    finish: float = 0.0
    x: np.ndarray | None = None
    iterations: int = 0
    status: int = -1
    residual: float = float("nan")
    error: str = ""                # why a request failed (its matrix could not be admitted)

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


@dataclass
class _Lane:
    """One k-slot batch of a resident matrix on its own engine (CUDA stream)."""
    eng: native.Engine
    factor: native.DeviceFactor
    op: native.DeviceOperator
    batch: native.Batch
    bbuf: list                     # pinned right-hand-side staging per slot
    xbuf: list                     # pinned solution staging per slot
    slots: list                    # live Request per slot, or None
    first_step: list               # first step id whose states show the slot's request
    staging: list = field(default_factory=list)        # (Request, future of its b copy) per slot, or None
    inflight: collections.deque = field(default_factory=collections.deque)   # step ids not yet consumed
    retiring: list = field(default_factory=list)       # [slot, Request, future of the x copy or None]
    next_step: int = 0

    def free(self, s: int) -> bool:
        return self.slots[s] is None and self.staging[s] is None

    def busy(self) -> bool:
        return bool(self.retiring) or bool(self.inflight) or any(s is not None for s in self.slots) or \
            any(s is not None for s in self.staging)

    def close(self):
        self.batch.close(); self.op.close(); self.factor.close(); self.eng.close()


@dataclass
class _Resident:
    mid: object
    n: int
    nbytes: int
    lanes: list
    queue: collections.deque = field(default_factory=collections.deque)
    last_used: float = 0.0

    def busy(self) -> bool:
        return bool(self.queue) or any(ln.busy() for ln in self.lanes)

    def close(self):
        for ln in self.lanes:
            ln.close()


def estimate_bytes(n: int, nnz_factor: int, nnz_a: int, k: int) -> int:
    """Upper estimate of the device bytes of one resident matrix: three pairs
    of factor arrays -- the factor's two sweep plans (entries + 32-position
    items), its canonical CSC / CSR (kept on the device for batch plans when
    it was prepared there) and the batch's two plans -- the fp32 sweep
    vectors, the permuted operator with its PCG vectors, and the batch's
    k-slot vectors (six fp64, three fp32) with its SpMV sub-tile partials
    (k * k / 2 doubles per 2048 rows)."""
    plan = 6 * (nnz_factor * 8 + n * 4 * 6)
    operator = nnz_a * 12 + n * (4 + 8 * 7)
    batch = n * k * (8 * 6 + 4 * 3) + n * 8 + (n // 2048 + 1) * max(1, k // 2) * k * 8
    return int(1.25 * (plan + operator + batch)) + (4 << 20)


class SolveServer:
    """Continuous-batching solve server on one GPU.

    register(mid, matrix, factor) makes a matrix known; submit(mid, b, tol)
    queues a request (admitting the matrix under the budget if needed);
    pump() advances every resident matrix once without blocking; drain()
    pumps until every request is done; run_open_loop(arrivals) submits
    requests at their arrival times while serving."""

    def __init__(self, device: int = 0, budget_bytes: int = 60 * 10**9, k: int = 8, iters_per_step: int = 2,
                 max_iter: int = 500, depth: int = 2, lanes: int = 1, sweep_grid: int | None = None,
                 copy_threads: int = 4, refresh_every: int | None = None):
        self.device, self.budget, self.k = device, int(budget_bytes), k
        # batches (streams) per matrix, and the sweep grid of each: None = the
        # resident grid divided among min(4, registered matrices x lanes), so the
        # latency-bound sweeps of different matrices run side by side instead of
        # each holding every SM; 0 = the resident grid; > 0 = that many blocks
        self.n_lanes, self.sweep_grid = max(1, lanes), sweep_grid
        self.refresh_every = refresh_every   # fp64 residual refresh period (None: the library default)
        # host copies of right-hand sides into pinned staging and of solutions out of it run on
        # worker threads (numpy releases the GIL for bulk copies), off the pump loop
        self.pool = concurrent.futures.ThreadPoolExecutor(copy_threads) if copy_threads > 0 else None
        self.iters_per_step, self.max_iter = iters_per_step, max_iter
        self.depth = max(1, min(2, depth))      # steps kept queued per matrix (the batch keeps two state copies)
        self.resident: dict = {}
        self.pending: dict = {}          # mid -> [future of its _Resident, reserved bytes, queued requests]
        # matrices are built (host preparation, uploads) on a worker thread while the pump keeps serving
        self.admitter = concurrent.futures.ThreadPoolExecutor(1)
        self.catalog: dict = {}          # mid -> (matrix, factor) that can be (re)admitted
        self.completed: list = []
        self.evictions = 0
        self.admissions = 0
        self._rid = 0

    # ---- matrices ----
    def register(self, mid, mat, fac):
        """Make a matrix known to the server (admitted to the device on first use)."""
        self.catalog[mid] = (mat, fac)

    def estimate(self, mid) -> int:
        mat, fac = self.catalog[mid]
        return self.n_lanes * estimate_bytes(mat.n, fac.nnz, mat.nnz, self.k)

    def used_bytes(self) -> int:
        """Bytes reserved by resident matrices (each: the larger of its estimate and its measured
        use) and by matrices being admitted (their estimate)."""
        return sum(r.nbytes for r in self.resident.values()) + sum(p[1] for p in self.pending.values())

    def _reserve(self, mid) -> int:
        """Make room for mid under the budget (evicting idle matrices, least
        recently used first); returns the bytes reserved."""
        need = self.estimate(mid)
        while self.used_bytes() + need > self.budget:
            idle = [r for r in self.resident.values() if not r.busy()]
            if not idle:
                raise BudgetError(f"matrix {mid!r} needs {need} bytes; {self.used_bytes()} of {self.budget} in use "
                                  "by busy matrices")
            victim = min(idle, key=lambda r: r.last_used)
            self.evict(victim.mid)
        return need

    def admit_matrix(self, mid):
        """Admit a matrix now (waits for an admission already under way)."""
        if mid in self.resident:
            return self.resident[mid]
        if mid in self.pending:
            self.pending[mid][0].result()
            self._collect_admissions()
            return self.resident[mid]
        need = self._reserve(mid)
        r = self._build(mid, need, self.budget - self.used_bytes())
        self.resident[mid] = r
        self.admissions += 1
        return r

    def _build(self, mid, need: int, room: int) -> _Resident:
        """The lanes of one matrix (engines, factor, operator, batch): room is
        the device budget its engines may use."""
        mat, fac = self.catalog[mid]
        import torch   # pinned host staging (page-locked buffers make the copies asynchronous)
        grid = self.sweep_grid
        if grid is None:
            parts = min(4, max(1, len(self.catalog)) * self.n_lanes)
            grid = 0 if parts == 1 else max(1, 2 * torch.cuda.get_device_properties(self.device).multi_processor_count
                                                // parts)
        lanes = []
        try:
            for _ in range(self.n_lanes):
                lanes.append(self._make_lane(mat, fac, grid, room + need - sum(ln.eng.memory_used() for ln in lanes)))
        except Exception:
            for ln in lanes:
                ln.close()
            raise
        used = sum(ln.eng.memory_used() for ln in lanes)
        return _Resident(mid=mid, n=mat.n, nbytes=max(need, used), lanes=lanes, last_used=time.perf_counter())

    def _collect_admissions(self) -> bool:
        """Make the matrices whose admission finished resident, with their queued requests."""
        progressed = False
        for mid in [m for m, p in self.pending.items() if p[0].done()]:
            fut, need, queue = self.pending.pop(mid)
            progressed = True
            try:
                r = fut.result()
            except Exception as ex:   # the requests of a matrix that could not be admitted fail
                for req in queue:
                    req.status, req.finish, req.error = native.ERR_BUDGET, time.perf_counter(), str(ex)
                    self.completed.append(req)
                continue
            r.queue.extend(queue)
            self.resident[mid] = r
            self.admissions += 1
        return progressed

    def _make_lane(self, mat, fac, grid: int, budget: int) -> _Lane:
        import torch
        eng = native.Engine(self.device)
        eng.set_memory_budget(max(1, budget))   # the engine refuses what would overrun the budget
        eng.set_sweep_grid(grid)
        f = op = bt = None
        try:
            f = native.DeviceFactor(eng, fac, precision=native.PREC_FP32)
            op = native.DeviceOperator(eng, mat, fac.perm)
            bt = native.Batch(eng, [f], [op], self.k)
            if self.refresh_every is not None:
                bt.set_refresh(self.refresh_every)
            bbuf = [torch.empty(mat.n, dtype=torch.float64).pin_memory().numpy() for _ in range(self.k)]
            xbuf = [torch.empty(mat.n, dtype=torch.float64).pin_memory().numpy() for _ in range(self.k)]
        except Exception as ex:
            for o in (bt, op, f, eng):
                if o is not None:
                    o.close()
            if isinstance(ex, native.ApxbError) and ex.code == native.ERR_BUDGET:
                raise BudgetError(str(ex)) from ex
            raise
        eng.set_sweep_grid(0)
        return _Lane(eng=eng, factor=f, op=op, batch=bt, bbuf=bbuf, xbuf=xbuf, slots=[None] * self.k,
                     first_step=[0] * self.k, staging=[None] * self.k)

    def evict(self, mid):
        r = self.resident[mid]
        if r.busy():
            raise RuntimeError("cannot evict a matrix with requests in flight")
        del self.resident[mid]
        r.close()
        self.evictions += 1

    # ---- requests ----
    def submit(self, mid, b, tol: float = 1e-8, arrival: float | None = None) -> Request:
        if mid not in self.catalog:
            raise KeyError(f"unknown matrix {mid!r}")
        self._rid += 1
        req = Request(rid=self._rid, mid=mid, b=np.ascontiguousarray(b, np.float64), tol=tol,
                      arrival=time.perf_counter() if arrival is None else arrival)
        if mid in self.resident:
            self.resident[mid].queue.append(req)
        elif mid in self.pending:
            self.pending[mid][2].append(req)
        else:
            # admission on a worker thread; the request waits in the admission's queue
            need = self._reserve(mid)
            room = self.budget - self.used_bytes()
            self.pending[mid] = [self.admitter.submit(self._build, mid, need, room), need,
                                 collections.deque([req])]
        return req

    def _run(self, fn, *args):
        if self.pool is None:
            f = concurrent.futures.Future()
            f.set_result(fn(*args))
            return f
        return self.pool.submit(fn, *args)

    @staticmethod
    def _copy_out(req, buf):
        req.x = buf.copy()
        req.finish = time.perf_counter()

    def _deliver(self, ln: _Lane, wait: bool = False) -> bool:
        """Start the host copy of every solution whose device copy has landed,
        and hand over the requests whose host copy is done."""
        progressed = False
        keep = []
        for ent in ln.retiring:
            s, req, fut = ent
            if fut is None and (wait or ln.batch.retired(s)):
                while not ln.batch.retired(s):
                    time.sleep(20e-6)
                fut = ent[2] = self._run(self._copy_out, req, ln.xbuf[s])
            if fut is not None and (wait or fut.done()):
                fut.result()
                self.completed.append(req)
                progressed = True
            else:
                keep.append(ent)
        ln.retiring = keep
        return progressed

    def _service(self, r: _Resident) -> bool:
        """One non-blocking pass over a resident matrix; returns whether anything happened.

        In every lane, steps stay queued on the device (up to `depth`) while
        the host reads the states of the oldest finished step, retires the slots
        that finished (their x copies are enqueued behind the queued steps) and
        admits waiting requests into the freed slots (they join at the next
        step once their right-hand side is staged). Waiting requests go to the
        lane with the most free slots."""
        progressed = False
        for ln in r.lanes:
            progressed |= self._deliver(ln)
            if ln.inflight and ln.batch.ready(ln.inflight[0]):
                sid = ln.inflight.popleft()
                progressed = True
                done, its, st, res = ln.batch.slots(sid)
                for s, req in enumerate(ln.slots):
                    if req is None or sid < ln.first_step[s] or not done[s]:
                        continue
                    if any(e[0] == s for e in ln.retiring):
                        self._deliver(ln, wait=True)       # the slot's previous solution is still in its buffer
                    req.iterations, req.status, req.residual = int(its[s]), int(st[s]), float(res[s])
                    ln.batch.retire(s, ln.xbuf[s])
                    ln.retiring.append([s, req, None])
                    ln.slots[s] = None
            # staged right-hand sides join the batch
            for s in range(self.k):
                stg = ln.staging[s]
                if stg is not None and stg[1].done():
                    stg[1].result()
                    req = stg[0]
                    ln.batch.admit(s, ln.bbuf[s], req.tol, self.max_iter)
                    ln.slots[s] = req
                    ln.first_step[s] = ln.next_step
                    ln.staging[s] = None
                    progressed = True
        while r.queue:
            ln = max(r.lanes, key=lambda x: sum(1 for q in range(self.k) if x.free(q)))
            free = [s for s in range(self.k) if ln.free(s)]
            if not free:
                break
            s = free[0]
            req = r.queue.popleft()
            req.start = time.perf_counter()
            ln.staging[s] = (req, self._run(np.copyto, ln.bbuf[s], req.b))
            progressed = True
        # keep the device busy
        for ln in r.lanes:
            while len(ln.inflight) < self.depth and any(x is not None for x in ln.slots):
                sid = ln.batch.step(self.iters_per_step)
                ln.next_step = sid + 1
                ln.inflight.append(sid)
                r.last_used = time.perf_counter()
                progressed = True
        return progressed

    def pump(self) -> bool:
        """Service every resident matrix once."""
        any_progress = self._collect_admissions()
        for r in list(self.resident.values()):
            any_progress |= self._service(r)
        return any_progress

    def idle(self) -> bool:
        return not self.pending and not any(r.busy() for r in self.resident.values())

    def drain(self, timeout: float = 600.0):
        t0 = time.perf_counter()
        while not self.idle():
            if not self.pump():
                time.sleep(20e-6)
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError("server did not drain")

    def run_open_loop(self, arrivals):
        """arrivals: list of (t_offset_seconds, mid, b, tol) sorted by time.
        Submits each at its time (open loop) while serving; returns the
        completed requests of this run."""
        start_n = len(self.completed)
        t0 = time.perf_counter()
        i = 0
        while i < len(arrivals) or not self.idle():
            now = time.perf_counter() - t0
            while i < len(arrivals) and arrivals[i][0] <= now:
                dt, mid, b, tol = arrivals[i]
                self.submit(mid, b, tol, arrival=t0 + dt)
                i += 1
            if not self.pump():
                time.sleep(20e-6)
        return self.completed[start_n:]

    def close(self):
        for mid in list(self.pending):
            try:
                self.pending[mid][0].result()
            except Exception:
                pass
        self._collect_admissions()
        self.admitter.shutdown(wait=True)
        for mid in list(self.resident):
            self.resident.pop(mid).close()
        if self.pool is not None:
            self.pool.shutdown(wait=True)
            self.pool = None


class MultiServer:
    """Requests routed by matrix id to one SolveServer per GPU (replicas, no
    collective): each registered matrix has one home device, which holds its
    factors, operator and batches; its requests go there. A matrix is placed
    on the device given at registration, else on the one with the fewest
    estimated bytes registered so far. The reference has one GPU path and no
    serving layer; this is the placement its solve phase allows (a triangular
    solve does not shard, the units -- matrices and their requests -- do)."""

    def __init__(self, devices, **server_kwargs):
        self.devices = list(devices)
        if not self.devices:
            raise ValueError("no devices")
        self.servers = [SolveServer(device=d, **server_kwargs) for d in self.devices]
        self.home: dict = {}                 # mid -> index into self.servers
        self.placed = [0] * len(self.servers)   # estimated bytes registered per device

    def register(self, mid, mat, fac, device=None):
        if mid in self.home:
            raise KeyError(f"matrix {mid!r} is already registered")
        if device is None:
            i = min(range(len(self.servers)), key=lambda j: (self.placed[j], j))
        else:
            i = self.devices.index(device)
        srv = self.servers[i]
        srv.register(mid, mat, fac)
        self.home[mid] = i
        self.placed[i] += srv.estimate(mid)
        return self.devices[i]

    def device_of(self, mid):
        return self.devices[self.home[mid]]

    def submit(self, mid, b, tol: float = 1e-8, arrival: float | None = None) -> Request:
        if mid not in self.home:
            raise KeyError(f"unknown matrix {mid!r}")
        return self.servers[self.home[mid]].submit(mid, b, tol, arrival)

    def pump(self) -> bool:
        progressed = False
        for srv in self.servers:
            progressed |= srv.pump()
        return progressed

    def idle(self) -> bool:
        return all(srv.idle() for srv in self.servers)

    def drain(self, timeout: float = 600.0):
        t0 = time.perf_counter()
        while not self.idle():
            if not self.pump():
                time.sleep(20e-6)
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError("servers did not drain")

    def run_open_loop(self, arrivals):
        """As SolveServer.run_open_loop, each request served on its matrix's device."""
        start = [len(srv.completed) for srv in self.servers]
        t0 = time.perf_counter()
        i = 0
        while i < len(arrivals) or not self.idle():
            now = time.perf_counter() - t0
            while i < len(arrivals) and arrivals[i][0] <= now:
                dt, mid, b, tol = arrivals[i]
                self.submit(mid, b, tol, arrival=t0 + dt)
                i += 1
            if not self.pump():
                time.sleep(20e-6)
        done = [q for srv, s0 in zip(self.servers, start) for q in srv.completed[s0:]]
        return sorted(done, key=lambda q: q.arrival)

    @property
    def completed(self):
        return [q for srv in self.servers for q in srv.completed]

    def close(self):
        for srv in self.servers:
            srv.close()


def latency_stats(reqs):
    lat = np.array([q.latency for q in reqs]) * 1e3
    if lat.size == 0:
        return {"count": 0}
    return {"count": int(lat.size), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
