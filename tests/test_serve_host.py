"""The solve server's host logic on CPU, with a fake batch in place of the
device: queueing, slot admission and retirement, asynchronous matrix
admission, the byte budget with least-recently-used eviction, and failed
admissions. (The device path is covered by tests/test_gpu_serve.py.)"""
import numpy as np
import pytest

from apxchol_b200 import native, serve
from apxchol_b200.serve import BudgetError, SolveServer, latency_stats


class _Mat:
    def __init__(self, n):
        self.n, self.nnz = n, 5 * n


class _Fac:
    def __init__(self, n):
        self.n, self.nnz = n, 4 * n


class _Closable:
    closed = False

    def close(self):
        self.closed = True

    def memory_used(self):
        return 1000


class FakeBatch(_Closable):
    """k slots; a slot admitted with b finishes after `need` iterations with x = 2 b."""

    def __init__(self, k, need=3):
        self.k, self.need = k, need
        self.b = [None] * k
        self.its = [0] * k
        self.live = [False] * k
        self.steps = []
        self.x = [None] * k

    def admit(self, s, b, tol, max_iter):
        assert not self.live[s]
        self.b[s], self.its[s], self.live[s] = np.array(b, copy=True), 0, True

    def step(self, iterations):
        for s in range(self.k):
            if self.live[s] and self.its[s] < self.need:
                self.its[s] = min(self.need, self.its[s] + iterations)
        state = ([self.live[s] and self.its[s] >= self.need for s in range(self.k)], list(self.its))
        self.steps.append(state)
        return len(self.steps) - 1

    def ready(self, sid):
        return True

    def slots(self, sid):
        done, its = self.steps[sid]
        n = self.k
        return np.array(done), np.array(its), np.zeros(n, np.int32), np.full(n, 1e-9)

    def retire(self, s, x):
        x[:] = 2.0 * self.b[s]
        self.live[s] = False
        return x

    def retired(self, s):
        return True


def _server(monkeypatch, budget=10**12, fail=()):
    made = []

    def make_lane(self, mat, fac, grid, room):
        if fac in fail:
            raise BudgetError("refused for the test")
        eng = _Closable()
        bt = FakeBatch(self.k)
        ln = serve._Lane(eng=eng, factor=_Closable(), op=_Closable(), batch=bt,
                         bbuf=[np.empty(mat.n) for _ in range(self.k)],
                         xbuf=[np.empty(mat.n) for _ in range(self.k)],
                         slots=[None] * self.k, first_step=[0] * self.k, staging=[None] * self.k)
        made.append(ln)
        return ln

    monkeypatch.setattr(SolveServer, "_make_lane", make_lane)
    srv = SolveServer(budget_bytes=budget, k=2, iters_per_step=1, sweep_grid=0, copy_threads=2)
    return srv, made


def test_requests_complete_with_their_own_results(monkeypatch):
    srv, _ = _server(monkeypatch)
    try:
        srv.register("a", _Mat(50), _Fac(50))
        srv.register("b", _Mat(70), _Fac(70))
        rng = np.random.default_rng(0)
        reqs = [srv.submit("ab"[j % 2], rng.standard_normal(50 if j % 2 == 0 else 70), 1e-8) for j in range(9)]
        srv.drain(timeout=30)
        assert len(srv.completed) == 9
        for q in reqs:
            assert q.status == 0 and q.iterations == 3
            assert np.array_equal(q.x, 2.0 * q.b)
            assert q.finish >= q.start >= q.arrival
        st = latency_stats(srv.completed)
        assert st["count"] == 9 and st["p99_ms"] >= st["p50_ms"]
        assert srv.admissions == 2 and srv.idle()
    finally:
        srv.close()


def test_budget_evicts_idle_and_refuses_busy(monkeypatch):
    srv, made = _server(monkeypatch)
    try:
        for mid in "abc":
            srv.register(mid, _Mat(100), _Fac(100))
        one = srv.estimate("a")
        srv.budget = one + one // 2          # one matrix at a time
        srv.admit_matrix("a")
        srv.admit_matrix("b")                # "a" idle: evicted
        assert set(srv.resident) == {"b"} and srv.evictions == 1 and made[0].eng.closed
        q = srv.submit("b", np.ones(100), 1e-8)       # "b" busy now
        with pytest.raises(BudgetError):
            srv.submit("c", np.ones(100), 1e-8)
        srv.drain(timeout=30)
        assert q.status == 0
        q2 = srv.submit("c", np.ones(100), 1e-8)      # "b" idle again: admitted on a worker thread
        assert "c" in srv.pending and srv.used_bytes() == one
        srv.drain(timeout=30)
        assert q2.status == 0 and set(srv.resident) == {"c"} and srv.evictions == 2
    finally:
        srv.close()


def test_failed_admission_fails_its_requests(monkeypatch):
    bad = _Fac(40)
    srv, _ = _server(monkeypatch, fail=(bad,))
    try:
        srv.register("ok", _Mat(40), _Fac(40))
        srv.register("bad", _Mat(40), bad)
        q_bad = srv.submit("bad", np.ones(40), 1e-8)
        q_ok = srv.submit("ok", np.ones(40), 1e-8)
        srv.drain(timeout=30)
        assert q_bad.status == native.ERR_BUDGET and q_bad.error and q_bad.x is None
        assert q_ok.status == 0
        assert "bad" not in srv.resident and srv.used_bytes() == srv.estimate("ok")
    finally:
        srv.close()


def test_open_loop_keeps_arrival_times(monkeypatch):
    srv, _ = _server(monkeypatch)
    try:
        srv.register("a", _Mat(30), _Fac(30))
        arrivals = [(0.001 * j, "a", np.full(30, float(j)), 1e-8) for j in range(12)]
        done = srv.run_open_loop(arrivals)
        assert len(done) == 12
        t0 = min(q.arrival for q in done)
        for q in done:
            assert q.finish >= q.arrival
            assert np.allclose(q.x, 2.0 * q.b)
        assert sorted(round(q.arrival - t0, 6) for q in done) == [round(0.001 * j, 6) for j in range(12)]
    finally:
        srv.close()


def test_multi_server_routes_by_matrix(monkeypatch):
    """MultiServer: each matrix gets one home device (the fewest estimated
    bytes so far, or the one given), its requests are served there and nowhere
    else, and every result is the request's own."""
    from apxchol_b200.serve import MultiServer

    def make_lane(self, mat, fac, grid, room):
        bt = FakeBatch(self.k)
        return serve._Lane(eng=_Closable(), factor=_Closable(), op=_Closable(), batch=bt,
                           bbuf=[np.empty(mat.n) for _ in range(self.k)],
                           xbuf=[np.empty(mat.n) for _ in range(self.k)],
                           slots=[None] * self.k, first_step=[0] * self.k, staging=[None] * self.k)

    monkeypatch.setattr(SolveServer, "_make_lane", make_lane)
    ms = MultiServer([0, 1, 2], budget_bytes=10**12, k=2, iters_per_step=1, sweep_grid=0, copy_threads=2)
    try:
        sizes = {"a": 50, "b": 70, "c": 60, "d": 40}
        for mid, n in sizes.items():
            ms.register(mid, _Mat(n), _Fac(n))
        assert [ms.device_of(m) for m in "abcd"] == [0, 1, 2, 0]
        assert ms.register("e", _Mat(10), _Fac(10), device=2) == 2
        rng = np.random.default_rng(3)
        reqs = []
        for j in range(15):
            mid = "abcde"[j % 5]
            reqs.append(ms.submit(mid, rng.standard_normal(sizes.get(mid, 10)), 1e-8))
        ms.drain(timeout=30)
        for q in reqs:
            assert q.status == 0 and np.array_equal(q.x, 2.0 * q.b)
        assert set(ms.servers[0].resident) == {"a", "d"}
        assert set(ms.servers[1].resident) == {"b"}
        assert set(ms.servers[2].resident) == {"c", "e"}
        assert len(ms.completed) == 15 and ms.idle()
        with pytest.raises(KeyError):
            ms.submit("zz", np.ones(3), 1e-8)
    finally:
        ms.close()
