"""Parity at the benchmark sizes (gpu).

The headline workload is the 3D 7-point 128^3 high-contrast SDDM grid
(n = 2,097,152, 176 sweep levels), factored by the reference with seed 1 on 8
threads -- the system bench.py times. On it:
  * the fp64 sweep pair is the reference omp_sptrsv's forward + transpose
    solve, bit for bit;
  * apxb_pcg takes the reference cpu_solver's iteration count +-2 and reaches
    the fp64-recomputed tolerance;
  * the batched mixed-precision form (k = 16, fp32 sweeps, fp64 outer) brings
    every slot to the fp64-recomputed relative residual tol, and each
    solution's error against the reference's FP64 solution of the same system
    is reported and bounded.
Then short cases at the other configurations' sizes: one R-MAT scale-22
Laplacian solve (iterations against the reference) and a sample of the
uneven multi-instance workload.

These take tens of seconds each (mostly the reference's CPU solves and the
factorizations).
"""
import numpy as np
import pytest

from apxchol_b200 import gen, native, workloads

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) absent")]

TOL = 1e-8
TRUE_RES_FACTOR = 10.0   # plain fp64 path: the recurrence residual stops it, fp64 drift allowed (test_gpu_pcg.py)
# Batched slots stop on a residual recomputed as b - A x in fp64 (the refresh that verifies convergence), so
# the host's own recomputation may differ from tol only by the rounding of the two computations.
HOST_RECOMPUTE_SLACK = 1.01
# ||x - x_ref|| / ||x_ref|| of a solve at relres 1e-8 against the reference's solve at relres 1e-8: each may
# be up to cond(A) * 1e-8 from the exact solution in the worst case; this bound is what the high-contrast
# 128^3 system shows with margin.
ORACLE_ERR_BOUND = 1e-5


def _true_res(A, b, x):
    return float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def grid128():
    A, F = workloads.grid3d_128()
    oracle.set_threads(oracle.host_cores())
    R = oracle.Ref(A, F)
    return A, F, R


def test_grid128_fp64_pair_is_the_reference_sweep(eng, grid128):
    import torch
    A, F, R = grid128
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    try:
        assert D.m == R.m == A.n and D.info.nnz_stored == R.nnz_stored
        assert D.info.fwd_levels == R.fwd_levels
        x = np.random.default_rng(21).standard_normal(D.m)
        y_ref = R.forward(x)
        z_ref = R.transpose(y_ref)
        dx = torch.from_numpy(x).cuda()
        dy = torch.empty_like(dx)
        D.sweep(0, dx, dy)
        eng.sync()
        assert np.array_equal(dy.cpu().numpy(), y_ref)
        dz = torch.empty_like(dx)
        D.sweep_pair(dx, dz)
        eng.sync()
        assert np.array_equal(dz.cpu().numpy(), z_ref)
    finally:
        D.close()


def test_grid128_pcg_matches_reference_iterations(eng, grid128):
    A, F, R = grid128
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    Op = native.DeviceOperator(eng, A, F.perm)
    try:
        for seed in (1000, 1001):
            b = gen.rhs(A.n, seed, False)
            xr, itr, _, _ = R.solve(b, TOL, 500)
            x, res = native.pcg(eng, D, Op, b, tol=TOL, max_iter=500)
            assert res.status == 0 and abs(res.iterations - itr) <= 2, (res.iterations, itr)
            assert _true_res(A, b, x) < TRUE_RES_FACTOR * TOL
            err = np.linalg.norm(x - xr) / np.linalg.norm(xr)
            print(f"grid3d_128 plain fp64 seed {seed}: {res.iterations} it (reference {itr}), "
                  f"error vs reference {err:.2e}")
            assert err <= ORACLE_ERR_BOUND, err
    finally:
        Op.close()
        D.close()


def test_grid128_batched_k16_every_slot_at_tol(eng, grid128):
    A, F, R = grid128
    k = 16
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    Op = native.DeviceOperator(eng, A, F.perm)
    bt = native.Batch(eng, [D], [Op], k)
    try:
        B = np.stack([gen.rhs(A.n, 1000 + c, False) for c in range(k)])
        xs, res = bt.solve([B], tol=TOL)
        errs, its_ref = [], []
        for c in range(k):
            r = res[0][c]
            assert r.status == 0, (c, r.status)
            assert r.true_residual <= TOL, (c, r.true_residual)
            assert _true_res(A, B[c], xs[0][c]) <= HOST_RECOMPUTE_SLACK * TOL, c
            if c < 4:   # the reference's FP64 solution of the same system (a CPU solve each)
                xr, itr, _, _ = R.solve(B[c], TOL, 500)
                errs.append(float(np.linalg.norm(xs[0][c] - xr) / np.linalg.norm(xr)))
                its_ref.append(itr)
        print(f"grid3d_128 batched k=16: iterations {[r.iterations for r in res[0]]}, reference {its_ref}, "
              f"FP64-oracle error {['%.2e' % e for e in errs]}")
        assert max(errs) <= ORACLE_ERR_BOUND, errs
    finally:
        bt.close()
        Op.close()
        D.close()


@pytest.fixture(scope="module")
def rmat22():
    return workloads.rmat_22()


def test_rmat22_solves_match_reference_iterations(eng, rmat22):
    """R-MAT scale 22 (a singular power-law Laplacian with hub rows of 10^5
    entries): one plain fp64 solve against the reference's iterations, and one
    batched mixed-precision pass of 4 right-hand sides at the fp64-recomputed
    tolerance."""
    A, F = rmat22
    oracle.set_threads(oracle.host_cores())
    R = oracle.Ref(A, F)
    b = gen.rhs(A.n, 3000, True)
    xr, itr, _, _ = R.solve(b, TOL, 500)
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    Op = native.DeviceOperator(eng, A, F.perm)
    try:
        x, res = native.pcg(eng, D, Op, b, tol=TOL, max_iter=500)
        assert res.status == 0 and abs(res.iterations - itr) <= 2, (res.iterations, itr)
        assert _true_res(A, b, x) < TRUE_RES_FACTOR * TOL
        assert abs(x.mean()) < 1e-10 * np.abs(x).max()
        err = float(np.linalg.norm(x - xr) / np.linalg.norm(xr))
        print(f"rmat_22 plain fp64: {res.iterations} it (reference {itr}), error vs reference {err:.2e}")
        assert err <= ORACLE_ERR_BOUND, err
    finally:
        D.close()
    D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    bt = native.Batch(eng, [D32], [Op], 4)
    try:
        B = np.stack([gen.rhs(A.n, 3000 + c, True) for c in range(4)])
        xs, bres = bt.solve([B], tol=TOL)
        for c in range(4):
            assert bres[0][c].status == 0 and bres[0][c].true_residual <= TOL, (c, bres[0][c].true_residual)
            assert _true_res(A, B[c], xs[0][c]) <= HOST_RECOMPUTE_SLACK * TOL
        err = float(np.linalg.norm(xs[0][0] - xr) / np.linalg.norm(xr))
        print(f"rmat_22 batched k=4: iterations {[r.iterations for r in bres[0]]}, FP64-oracle error {err:.2e}")
        assert err <= ORACLE_ERR_BOUND, err
    finally:
        bt.close()
        D32.close()
        Op.close()


def test_instances_sample_in_one_batch(eng):
    """The first 24 instances of the uneven multi-instance workload (n uniform
    in [1000, 200000], 2D grids and 6-regular graphs, 1-8 right-hand sides
    each) in one batch: every slot at the fp64-recomputed tolerance, and the
    reference's iterations and solution for one right-hand side of each."""
    insts = workloads.instances_256(count=24)
    Ds = [native.DeviceFactor(eng, F, precision=native.PREC_FP32) for _, F, _ in insts]
    Ops = [native.DeviceOperator(eng, A, F.perm) for A, F, _ in insts]
    bt = native.Batch(eng, Ds, Ops, 8)
    try:
        rhs = [np.stack([gen.rhs(A.n, 5000 + 10 * i + j, False) for j in range(c)])
               for i, (A, F, c) in enumerate(insts)]
        xs, res = bt.solve(rhs, tol=TOL)
        oracle.set_threads(oracle.host_cores())
        worst = 0.0
        for i, (A, F, c) in enumerate(insts):
            for j in range(c):
                r = res[i][j]
                assert r.status == 0 and r.true_residual <= TOL, (i, j, r.status, r.true_residual)
                assert _true_res(A, rhs[i][j], xs[i][j]) <= HOST_RECOMPUTE_SLACK * TOL, (i, j)
            xr, itr, _, _ = oracle.Ref(A, F).solve(rhs[i][0], TOL, 500)
            worst = max(worst, float(np.linalg.norm(xs[i][0] - xr) / np.linalg.norm(xr)))
            assert abs(res[i][0].iterations - itr) <= 5, (i, res[i][0].iterations, itr)
        print(f"instances sample: {len(insts)} instances, FP64-oracle error max {worst:.2e}")
        assert worst <= ORACLE_ERR_BOUND, worst
    finally:
        bt.close()
        for o in Ops + Ds:
            o.close()
