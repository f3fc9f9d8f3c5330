"""GPU-resident PCG against the reference cpu_solver (gpu): iterations within
+-2 of the reference, the fp64-recomputed relative residual at tol, the
solution within the PCG tolerance of the reference's (after null-space
centring for Laplacians), and bit-identical repeated solves."""
import numpy as np
import pytest

from apxchol_b200 import gen, native
from tests import golden_cases as gc
from tests.problems import problem

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-8
TRUE_RES_FACTOR = 10.0   # true residual may exceed the recurrence residual by fp64 drift


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def _true_res(A, b, x):
    return np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b)


@pytest.mark.parametrize("name", gc.NAMES)
def test_pcg_matches_reference_golden(eng, name):
    A, F, g = gc.case(name)
    D = native.DeviceFactor(eng, F)
    Op = native.DeviceOperator(eng, A, F.perm)
    x, res = native.pcg(eng, D, Op, g["b"], tol=TOL, max_iter=500)
    assert abs(res.iterations - int(g["pcg_iters"])) <= 2
    assert res.status == 0 and res.residual < TOL
    assert res.true_residual < TRUE_RES_FACTOR * TOL
    assert _true_res(A, g["b"], x) < TRUE_RES_FACTOR * TOL
    if not F.sddm:
        assert abs(x.mean()) < 1e-12 * np.abs(x).max()
    xr = g["pcg_x"]
    assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_48", "regular_3000", "rmat_12", "rmat_14"])
def test_pcg_matches_oracle_and_repeats_bitwise(eng, name):
    """rmat_12 / rmat_14 have operator rows longer than the long-row threshold
    (128 entries), so their SpMV takes the chunked path."""
    A, F = problem(name)
    O = oracle.Oracle(A, F, nt=8)
    D = native.DeviceFactor(eng, F)
    Op = native.DeviceOperator(eng, A, F.perm)
    b = gen.rhs(A.n, 9, not F.sddm)
    xo, ito, reso = O.solve(b, TOL, 500)
    x1, r1 = native.pcg(eng, D, Op, b, tol=TOL, max_iter=500)
    x2, r2 = native.pcg(eng, D, Op, b, tol=TOL, max_iter=500)
    assert abs(r1.iterations - ito) <= 2, (r1.iterations, ito)
    assert r1.true_residual < TRUE_RES_FACTOR * TOL
    assert np.array_equal(x1, x2) and r1.iterations == r2.iterations
    assert np.linalg.norm(x1 - xo) <= 1e-6 * np.linalg.norm(xo)


def test_pcg_edge_cases(eng):
    A, F = problem("grid2d_64")
    D = native.DeviceFactor(eng, F)
    Op = native.DeviceOperator(eng, A, F.perm)
    # zero rhs: x = 0, no iterations (src/solve.cpp:544-545)
    x, r = native.pcg(eng, D, Op, np.zeros(A.n), tol=TOL, max_iter=50)
    assert r.iterations == 0 and not x.any()
    # max_iter cap
    b = gen.rhs(A.n, 1, True)
    x, r = native.pcg(eng, D, Op, b, tol=1e-30, max_iter=3)
    assert r.iterations == 3 and r.status == 1
    # a non-finite rhs ends with status 4 (non-finite), not a hang
    bn = b.copy(); bn[5] = np.nan
    x, r = native.pcg(eng, D, Op, bn, tol=TOL, max_iter=20)
    assert r.status == 4
    # and the engine keeps working
    x, r = native.pcg(eng, D, Op, b, tol=TOL, max_iter=500)
    assert r.status == 0


def test_fp32_exact_operator_is_stored_in_fp32(eng, monkeypatch):
    """An operator whose values are all fp32-exact is stored in fp32 (the
    reference's rule, pcg_cuda.h:100-111) and solves to the same bits as the
    same operator stored in fp64 (APXCHOL_GPU_FP32_OPERATOR=0): the SpMV widens
    every value to fp64 either way. Plain PCG, and batches of one instance, of
    two fp32 instances and of a mixed pair (combined operator widened)."""
    from apxchol_b200 import refsetup
    from apxchol_b200.gen import Matrix
    A0, F0 = problem("grid2d_64")
    assert not native.DeviceOperator(eng, A0, F0.perm).fp32
    # the same Laplacian with weights rounded to multiples of 1/8: every value,
    # diagonal sums included, is exact in fp32
    cols = np.repeat(np.arange(A0.n), np.diff(A0.colptr))
    diag = A0.rowidx == cols
    vals = np.where(diag, 0.0, -np.round(np.abs(A0.vals) * 8.0) / 8.0)
    vals[diag] = -np.bincount(cols, weights=vals, minlength=A0.n)[cols[diag]]
    assert np.array_equal(vals, vals.astype(np.float32).astype(np.float64))
    A = Matrix(n=A0.n, colptr=A0.colptr, rowidx=A0.rowidx, vals=vals, name="grid2d_64_f32", sddm=A0.sddm)
    F = refsetup.factorize(A, seed=0, threads=refsetup.DEFAULT_THREADS)
    D = native.DeviceFactor(eng, F)
    Op32 = native.DeviceOperator(eng, A, F.perm)
    monkeypatch.setenv("APXCHOL_GPU_FP32_OPERATOR", "0")
    Op64 = native.DeviceOperator(eng, A, F.perm)
    monkeypatch.delenv("APXCHOL_GPU_FP32_OPERATOR")
    assert Op32.fp32 and not Op64.fp32
    b = gen.rhs(A.n, 31, not F.sddm)
    x32, r32 = native.pcg(eng, D, Op32, b, tol=TOL, max_iter=500)
    x64, r64 = native.pcg(eng, D, Op64, b, tol=TOL, max_iter=500)
    assert r32.status == 0 and r32.iterations == r64.iterations
    assert np.array_equal(x32, x64)
    assert np.array_equal(Op32.matvec(b), Op64.matvec(b))
    D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    B = np.stack([gen.rhs(A.n, 40 + c, not F.sddm) for c in range(4)])
    out = []
    for ops in ([Op32], [Op64], [Op32, Op32], [Op32, Op64]):
        bt = native.Batch(eng, [D32] * len(ops), ops, 4)
        out.append(bt.solve([B] * len(ops), tol=TOL)[0])
        bt.close()
    for o in out:
        for xi in o:
            assert np.array_equal(xi, out[0][0])
