"""Serving (gpu): continuous batching over resident factors.

A request's result is the same alone and in the mix -- bit for bit: every
slot's arithmetic is independent of the other slots and of its slot index,
so the tolerance here is zero. Requests that arrive while others run are
admitted at iteration boundaries; matrices are admitted under a device
memory budget with least-recently-used eviction of idle ones."""
import numpy as np
import pytest

from apxchol_b200 import gen, native
from apxchol_b200.serve import BudgetError, SolveServer, latency_stats
from tests.problems import problem

pytestmark = pytest.mark.gpu
K = 4
TRUE_RES_FACTOR = 10.0


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    torch.cuda.init()


def _alone(mat, fac, b, tol, refresh=None):
    """The same right-hand side solved by itself (one slot of a fresh batch)."""
    eng = native.Engine(0)
    try:
        D = native.DeviceFactor(eng, fac, precision=native.PREC_FP32)
        Op = native.DeviceOperator(eng, mat, fac.perm)
        bt = native.Batch(eng, [D], [Op], K)
        if refresh is not None:
            bt.set_refresh(refresh)
        xs, res = bt.solve([b[None, :]], tol=tol)
        out = xs[0][0].copy(), res[0][0]
        bt.close(); Op.close(); D.close()
        return out
    finally:
        eng.close()


@pytest.mark.parametrize("lanes,refresh", [(1, None), (2, None), (1, 3)])
def test_results_equal_alone_and_in_the_mix(lanes, refresh):
    """refresh = 3: the periodic fp64 residual refresh runs every 3 iterations of
    each slot, at different batch iterations for different slots."""
    mats = {"g2": problem("grid2d_64"), "g3": problem("grid3d_24"), "rr": problem("regular_3000")}
    srv = SolveServer(k=K, iters_per_step=3, lanes=lanes, refresh_every=refresh)
    try:
        for mid, (A, F) in mats.items():
            srv.register(mid, A, F)
        reqs = []
        tols = [1e-6, 1e-8, 1e-10]
        # staggered: submit some, let them run, submit more while they are in flight
        order = ["g2", "g3", "rr", "g3", "g2", "g3", "rr", "rr", "g2", "g3", "g3", "g2", "rr"]
        for j, mid in enumerate(order):
            A, F = mats[mid]
            b = gen.rhs(A.n, 200 + j, not F.sddm)
            reqs.append(srv.submit(mid, b, tols[j % 3]))
            if j % 4 == 3:
                for _ in range(3):
                    srv.pump()
        srv.drain()
        assert len(srv.completed) == len(order)
        for req in reqs:
            A, F = mats[req.mid]
            x_alone, r_alone = _alone(A, F, req.b, req.tol, refresh)
            assert req.status == 0, (req.mid, req.status)
            assert np.array_equal(req.x, x_alone), req.rid
            assert req.iterations == r_alone.iterations
            relres = np.linalg.norm(req.b - A.matvec(req.x)) / np.linalg.norm(req.b)
            assert relres < TRUE_RES_FACTOR * req.tol, (req.rid, relres, req.tol)
        st = latency_stats(srv.completed)
        assert st["count"] == len(order) and st["p99_ms"] >= st["p50_ms"] > 0
    finally:
        srv.close()


def test_open_loop_arrivals():
    A, F = problem("grid2d_64")
    srv = SolveServer(k=K, iters_per_step=2)
    try:
        srv.register("g", A, F)
        rng = np.random.default_rng(1)
        t = np.cumsum(rng.exponential(1 / 400.0, size=24))
        arrivals = [(float(t[j]), "g", gen.rhs(A.n, 900 + j, True), 1e-8) for j in range(24)]
        done = srv.run_open_loop(arrivals)
        assert len(done) == 24 and all(q.status == 0 for q in done)
        assert all(q.finish >= q.start >= q.arrival for q in done)
    finally:
        srv.close()


def test_budget_admission_and_eviction():
    A1, F1 = problem("grid2d_64")
    A2, F2 = problem("grid3d_24")
    srv = SolveServer(k=K)
    try:
        srv.register("a", A1, F1)
        srv.register("b", A2, F2)
        ea, eb = srv.estimate("a"), srv.estimate("b")
        srv.budget = max(ea, eb) + min(ea, eb) // 2     # room for one matrix only
        srv.admit_matrix("a")
        assert srv.resident["a"].lanes[0].eng.memory_used() <= ea == srv.used_bytes()
        srv.admit_matrix("b")                # evicts idle "a"
        assert "a" not in srv.resident and srv.evictions == 1
        assert srv.resident["b"].lanes[0].eng.memory_used() <= eb == srv.used_bytes()
        req = srv.submit("b", gen.rhs(A2.n, 1, False), 1e-8)   # "b" busy
        with pytest.raises(BudgetError):
            srv.admit_matrix("a")            # cannot evict a busy matrix
        srv.drain()
        assert req.status == 0
        srv.admit_matrix("a")                # "b" idle again: evicted
        assert set(srv.resident) == {"a"}
    finally:
        srv.close()


def test_slot_primitives():
    A, F = problem("grid2d_64")
    eng = native.Engine(0)
    try:
        D = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
        Op = native.DeviceOperator(eng, A, F.perm)
        bt = native.Batch(eng, [D], [Op], 2)
        with pytest.raises(native.ApxbError):
            bt.step(1)                       # nothing admitted yet
        b = gen.rhs(A.n, 7, True)
        bt.admit(0, b, 1e-8)
        with pytest.raises(native.ApxbError) as ex:
            bt.admit(0, b, 1e-8)             # slot 0 is admitted
        assert ex.value.code == native.ERR_BUSY
        with pytest.raises(native.ApxbError) as ex:
            bt.solve([b[None, :]], tol=1e-8)   # a whole-batch solve waits for the slots
        assert ex.value.code == native.ERR_BUSY
        sids = []
        for _ in range(200):
            sids.append(bt.step(5))
            done, its, st, res = bt.slots(sids[-1])
            if done[0]:
                break
        assert done[0] and st[0] == 0 and done[1]      # slot 1 was never admitted: idle
        if len(sids) >= 3:
            with pytest.raises(native.ApxbError):
                bt.slots(sids[-3])           # only the last two steps' states are kept
        x = bt.retire(0)
        assert bt.retired(0)
        xs, _ = bt.solve([b[None, :]], tol=1e-8)
        assert np.array_equal(x, xs[0][0])
        bt.close(); Op.close(); D.close()
    finally:
        eng.close()
