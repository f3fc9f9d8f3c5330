"""Batched mixed-precision solves (gpu): many right-hand sides and uneven
instances in one set of launches. fp32 preconditioner sweeps, fp64 outer
PCG: every slot must reach the fp64-recomputed tolerance and agree with the
reference's solution within the PCG tolerance; batched results must equal
the same systems solved alone."""
import numpy as np
import pytest

from apxchol_b200 import gen, native
from tests.problems import problem

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-8
TRUE_RES_FACTOR = 10.0


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def _objs(eng, name):
    A, F = problem(name)
    return A, F, native.DeviceFactor(eng, F, precision=native.PREC_FP32), native.DeviceOperator(eng, A, F.perm)


@pytest.mark.parametrize("k", [1, 4, 16, 32, 64, 128])
def test_single_instance_multi_rhs(eng, k):
    A, F, D, Op = _objs(eng, "grid3d_24")
    bt = native.Batch(eng, [D], [Op], k)
    B = np.stack([gen.rhs(A.n, 100 + c, False) for c in range(k)])
    xs, res = bt.solve([B], tol=TOL)
    O = oracle.Oracle(A, F, nt=8)
    for c in range(k):
        r = res[0][c]
        assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL, (c, r.status, r.true_residual)
        xo, ito, _ = O.solve(B[c], TOL, 500)
        assert np.linalg.norm(xs[0][c] - xo) <= 1e-6 * np.linalg.norm(xo)
        assert abs(r.iterations - ito) <= 5, (r.iterations, ito)


def test_uneven_instances_share_one_batch(eng):
    names = ["grid2d_64", "grid3d_24", "regular_3000", "rmat_12"]
    objs = [_objs(eng, nm) for nm in names]
    bt = native.Batch(eng, [o[2] for o in objs], [o[3] for o in objs], 4)
    rhs = []
    for i, (A, F, D, Op) in enumerate(objs):
        c = 1 + i % 4
        rhs.append(np.stack([gen.rhs(A.n, 10 * i + j, not F.sddm) for j in range(c)]))
    xs, res = bt.solve(rhs, tol=TOL)
    for i, (A, F, D, Op) in enumerate(objs):
        # each instance alone in its own batch gives the same bytes
        alone = native.Batch(eng, [D], [Op], 4)
        xa, ra = alone.solve([rhs[i]], tol=TOL)
        assert np.array_equal(xs[i], xa[0]), names[i]
        for c in range(rhs[i].shape[0]):
            r = res[i][c]
            assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL, (names[i], c, r.true_residual)
            assert r.iterations == ra[0][c].iterations
            if not F.sddm:
                assert abs(xs[i][c].mean()) < 1e-10 * np.abs(xs[i][c]).max()


def test_batch_repeats_bitwise(eng):
    A, F, D, Op = _objs(eng, "grid2d_256")
    bt = native.Batch(eng, [D], [Op], 8)
    B = np.stack([gen.rhs(A.n, 500 + c, True) for c in range(5)])
    x1, r1 = bt.solve([B], tol=TOL)
    x2, r2 = bt.solve([B], tol=TOL)
    assert np.array_equal(x1[0], x2[0])
    assert [r.iterations for r in r1[0]] == [r.iterations for r in r2[0]]


def test_autotuner_picks_the_fastest_candidate(eng):
    from apxchol_b200 import autotune
    A, F, D, Op = _objs(eng, "grid3d_24")
    ch = autotune.tune(eng, D, Op, lambda j: gen.rhs(A.n, 500 + j, False), ks=(1, 4), grids=(0, 64))
    assert len(ch.table) == 4
    assert ch.solves_per_s == max(t[2] for t in ch.table)
    assert (ch.k, ch.grid) in [(t[0], t[1]) for t in ch.table]


def test_lanes_give_the_same_bits_as_one_batch(eng):
    """Concurrent batches on separate streams (apxchol_b200.lanes) with a cut
    sweep grid return exactly what one batch returns."""
    import torch
    from apxchol_b200.lanes import Lanes
    A, F, D, Op = _objs(eng, "grid3d_24")
    k = 4
    B = np.stack([gen.rhs(A.n, 700 + c, False) for c in range(k)])
    bt = native.Batch(eng, [D], [Op], k)
    want, _ = bt.solve([B], tol=TOL)
    ln = Lanes(A, F, k, lanes=3)
    try:
        Bf, nrhs = ln.pack(B)
        Bs = [torch.from_numpy(Bf).cuda() for _ in range(3)]
        Xs = [torch.empty_like(b) for b in Bs]
        res = ln.solve_raw(Bs, Xs, nrhs, tol=TOL, flags=native.DEVICE_PTRS)
        for j in range(3):
            got = ln.lanes[j].batch.unpack(Xs[j].cpu().numpy(), nrhs)[0]
            assert np.array_equal(got, want[0])
            assert all(r.status == 0 for r in res[j][:k])
    finally:
        ln.close()


def _mixed_instances(count: int, seed: int):
    """SDDM instances shaped like the uneven multi-instance workload, scaled
    down: half 2D 5-point grids (weights U[1,2]), half random 6-regular graphs
    (weights U[0.5,2]), diagonal shift 1e-3 * degree, sizes drawn uniformly."""
    from apxchol_b200 import refsetup
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        if i % 2 == 0:
            side = int(rng.integers(20, 90))
            A = gen.grid2d(side, int(rng.integers(20, 90)), seed=100 + i, shift=1e-3)
        else:
            A = gen.random_regular(int(rng.integers(1000, 6000)), seed=100 + i, shift=1e-3)
        F = refsetup.factorize(A, seed=i, threads=8)
        out.append((A, F))
    return out


@pytest.mark.parametrize("k", [4, 8])
def test_many_uneven_instances_in_one_batch(eng, k):
    insts = _mixed_instances(24, seed=k)
    Ds = [native.DeviceFactor(eng, F, precision=native.PREC_FP32) for _, F in insts]
    Ops = [native.DeviceOperator(eng, A, F.perm) for A, F in insts]
    bt = native.Batch(eng, Ds, Ops, k)
    rng = np.random.default_rng(7)
    rhs = [np.stack([gen.rhs(A.n, 1000 * i + j, False) for j in range(int(rng.integers(1, k + 1)))])
           for i, (A, F) in enumerate(insts)]
    xs, res = bt.solve(rhs, tol=TOL)
    for i, (A, F) in enumerate(insts):
        for c in range(rhs[i].shape[0]):
            r = res[i][c]
            assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL, (i, c, r.true_residual)
            relres = np.linalg.norm(rhs[i][c] - A.matvec(xs[i][c])) / np.linalg.norm(rhs[i][c])
            assert relres < TRUE_RES_FACTOR * TOL
    # a few instances alone give the same bits
    for i in (0, 5, 23):
        alone = native.Batch(eng, [Ds[i]], [Ops[i]], k)
        xa, _ = alone.solve([rhs[i]], tol=TOL)
        assert np.array_equal(xs[i], xa[0]), i


def test_instance_autotuner(eng):
    from apxchol_b200 import autotune
    insts = _mixed_instances(6, seed=3)
    Ds = [native.DeviceFactor(eng, F, precision=native.PREC_FP32) for _, F in insts]
    Ops = [native.DeviceOperator(eng, A, F.perm) for A, F in insts]
    rhs = [np.stack([gen.rhs(A.n, 50 * i + j, False) for j in range(1 + i % 5)]) for i, (A, F) in enumerate(insts)]
    k, table = autotune.tune_instances(eng, Ds, Ops, rhs, ks=(1, 2, 4, 8))
    assert [t[0] for t in table] == [1, 2, 4, 8]
    assert k == max(table, key=lambda t: t[1])[0]


@pytest.mark.parametrize("k", [1, 4])
def test_long_operator_rows(eng, k):
    """Operator rows longer than the long-row threshold (128 entries; rmat_14
    has rows up to 3676) go through the chunked SpMV; the batch still
    converges, agrees with the reference's solution and repeats bit for bit."""
    A, F, D, Op = _objs(eng, "rmat_14")
    assert np.diff(A.colptr).max() > 2048
    bt = native.Batch(eng, [D], [Op], k)
    B = np.stack([gen.rhs(A.n, 300 + c, True) for c in range(k)])
    x1, r1 = bt.solve([B], tol=TOL)
    x2, r2 = bt.solve([B], tol=TOL)
    assert np.array_equal(x1[0], x2[0])
    O = oracle.Oracle(A, F, nt=8)
    for c in range(k):
        assert r1[0][c].status == 0 and r1[0][c].true_residual < TRUE_RES_FACTOR * TOL
        xo, ito, _ = O.solve(B[c], TOL, 500)
        assert np.linalg.norm(x1[0][c] - xo) <= 1e-6 * np.linalg.norm(xo)


@pytest.mark.parametrize("every", [0, 3])
def test_residual_refresh(eng, every):
    """The periodic fp64 residual refresh (r = b - A x every `every` iterations of
    a slot) keeps convergence and accuracy, and repeats bit for bit."""
    A, F, D, Op = _objs(eng, "grid3d_24")
    bt = native.Batch(eng, [D], [Op], 4)
    bt.set_refresh(every)
    B = np.stack([gen.rhs(A.n, 400 + c, False) for c in range(4)])
    x1, r1 = bt.solve([B], tol=TOL)
    x2, r2 = bt.solve([B], tol=TOL)
    assert np.array_equal(x1[0], x2[0])
    O = oracle.Oracle(A, F, nt=8)
    for c in range(4):
        assert r1[0][c].status == 0 and r1[0][c].true_residual < TRUE_RES_FACTOR * TOL
        xo, ito, _ = O.solve(B[c], TOL, 500)
        assert np.linalg.norm(x1[0][c] - xo) <= 1e-6 * np.linalg.norm(xo)


def _centred(x):
    return x - x.mean()


@pytest.mark.parametrize("k", [4, 16, 64])
def test_fp16_factor_storage_in_the_batch(eng, k):
    """The reference GPU path's default storage -- fp16 values of the
    column-scaled factor, a per-row fp32 diagonal, the backward input times
    (1/s)^2 in fp64 (cuda.h:131-163, cuda_dataflow.cu:395) -- in the batched
    sweeps. Every slot meets the true-residual gate and lies within the PCG
    tolerance of the reference's FP64 solution (the oracle); iterations stay
    within 3 of the fp32-stored factor's (fp16 rounds every off-diagonal to 11
    bits, a slightly different preconditioner)."""
    for name in ("grid3d_24", "grid2d_64"):
        A, F = problem(name)
        D16 = native.DeviceFactor(eng, F, precision=native.PREC_FP16)
        D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
        Op = native.DeviceOperator(eng, A, F.perm)
        B = np.stack([gen.rhs(A.n, 300 + c, not F.sddm) for c in range(k)])
        b16 = native.Batch(eng, [D16], [Op], k)
        x16, r16 = b16.solve([B], tol=TOL)
        x16b, _ = b16.solve([B], tol=TOL)
        assert np.array_equal(x16[0], x16b[0])            # repeats bitwise
        b32 = native.Batch(eng, [D32], [Op], k)
        _, r32 = b32.solve([B], tol=TOL)
        O = oracle.Oracle(A, F, nt=8)
        for c in range(k):
            r = r16[0][c]
            assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL, (name, c, r.status, r.true_residual)
            assert abs(r.iterations - r32[0][c].iterations) <= 3, (name, c, r.iterations, r32[0][c].iterations)
            if c < 8:
                xo, _, _ = O.solve(B[c], TOL, 500)
                assert np.linalg.norm(_centred(x16[0][c]) - _centred(xo)) <= 1e-6 * np.linalg.norm(_centred(xo))
        b16.close(); b32.close()


def test_fp16_instances_share_one_batch(eng):
    """fp16 instances of different sizes in one batch give each instance's
    bytes alone; a batch mixing fp16 and fp32 factors sweeps every instance
    over its fp32 values and still converges."""
    names = ["grid2d_64", "grid3d_24", "regular_3000"]
    objs = []
    for nm in names:
        A, F = problem(nm)
        objs.append((A, F, native.DeviceFactor(eng, F, precision=native.PREC_FP16),
                     native.DeviceFactor(eng, F, precision=native.PREC_FP32), native.DeviceOperator(eng, A, F.perm)))
    rhs = [np.stack([gen.rhs(A.n, 50 + 3 * i + j, not F.sddm) for j in range(1 + i)])
           for i, (A, F, _, _, _) in enumerate(objs)]
    bt = native.Batch(eng, [o[2] for o in objs], [o[4] for o in objs], 4)
    xs, res = bt.solve(rhs, tol=TOL)
    for i, (A, F, D16, D32, Op) in enumerate(objs):
        alone = native.Batch(eng, [D16], [Op], 4)
        xa, _ = alone.solve([rhs[i]], tol=TOL)
        assert np.array_equal(xs[i], xa[0]), names[i]
        for r in res[i]:
            assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL
    mixed = native.Batch(eng, [objs[0][2], objs[1][3]], [objs[0][4], objs[1][4]], 4)
    _, rm = mixed.solve(rhs[:2], tol=TOL)
    for ri in rm:
        for r in ri:
            assert r.status == 0 and r.true_residual < TRUE_RES_FACTOR * TOL
