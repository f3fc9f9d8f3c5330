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
