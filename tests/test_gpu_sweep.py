"""Parity of the CUDA sweeps with the reference arithmetic (gpu).

fp64 sweeps must reproduce the reference CPU sweep (omp_sptrsv) byte for
byte: same arrays, same per-row sum order, every product and sum rounded on
its own. The fp32 sweeps are checked against the fp64 result with a stated
tolerance."""
import numpy as np
import pytest

from apxchol_b200 import native
from tests import golden_cases as gc
from tests.problems import problem

import oracle

pytestmark = pytest.mark.gpu

FP32_SWEEP_RTOL = 1e-4   # fp32 factor values are exact; fp32 accumulation over the two sweeps


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _pair_dev(eng, D, x):
    import torch
    dx = _dev(x)
    dz = torch.empty_like(dx)
    torch.cuda.synchronize()
    D.sweep_pair(dx, dz)
    eng.sync()
    return dz.cpu().numpy()


@pytest.mark.parametrize("name", gc.NAMES)
def test_fp64_sweeps_match_reference_golden(eng, name):
    import torch
    A, F, g = gc.case(name)
    D = native.DeviceFactor(eng, F)
    dx = _dev(g["x"])
    dy = torch.empty_like(dx)
    torch.cuda.synchronize()
    D.sweep(0, dx, dy)
    eng.sync()
    assert np.array_equal(dy.cpu().numpy(), g["fwd"])
    dz = torch.empty_like(dx)
    D.sweep(1, dy, dz)
    eng.sync()
    assert np.array_equal(dz.cpu().numpy(), g["pair"])
    assert np.array_equal(_pair_dev(eng, D, g["x"]), g["pair"])
    assert np.array_equal(D.sweep_pair_host(g["x"]), g["pair"])


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_48", "regular_3000", "rmat_12", "path_200"])
def test_fp64_pair_matches_oracle_and_is_schedule_free(eng, name):
    A, F = problem(name)
    O = oracle.Oracle(A, F)
    D = native.DeviceFactor(eng, F)
    x = np.random.default_rng(2).standard_normal(F.m)
    want = O.pair(x)
    got = _pair_dev(eng, D, x)
    assert np.array_equal(got, want)
    # bit-identical run to run and for any grid (1 block, 7 blocks, resident)
    for grid in (1, 7, 0):
        eng.set_sweep_grid(grid)
        assert np.array_equal(_pair_dev(eng, D, x), want), grid
    eng.set_sweep_grid(0)


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_48", "regular_3000"])
def test_fp32_pair_within_tolerance(eng, name):
    A, F = problem(name)
    O = oracle.Oracle(A, F)
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    x = np.random.default_rng(3).standard_normal(F.m)
    want = O.pair(x)
    got = _pair_dev(eng, D, x)
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < FP32_SWEEP_RTOL, err
    assert np.array_equal(_pair_dev(eng, D, x), got)      # deterministic


@pytest.mark.parametrize("k", [1, 2, 4, 8, 16])
def test_fp32_multi_rhs_equals_single(eng, k):
    import torch
    A, F = problem("grid3d_24")
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    X = np.random.default_rng(4).standard_normal((F.m, k))
    dX = _dev(X)
    dZ = torch.empty_like(dX)
    torch.cuda.synchronize()
    D.sweep_pair_multi(k, dX, dZ)
    eng.sync()
    Z = dZ.cpu().numpy()
    for s in range(k):
        # same entry order and fp32 arithmetic per column: identical to a k=1 sweep
        assert np.array_equal(Z[:, s], _pair_dev(eng, D, X[:, s])), s


def test_apply_sddm_is_bit_exact_and_laplacian_close(eng):
    A, F, g = gc.case("grid3d_10")          # SDDM: no centring, every op exact
    D = native.DeviceFactor(eng, F)
    z, rz = D.apply(g["b"])
    assert np.array_equal(z, g["apply"])
    A, F, g = gc.case("grid2d_32")          # Laplacian: permute/gather exact, means differ in association
    D = native.DeviceFactor(eng, F)
    O = oracle.Oracle(A, F)
    for k in range(12):                     # the center-k schedule: only the 10th application centres
        z, rz = D.apply(g["b"])
        zo = O.apply(g["b"], reset=(k == 0))
        assert np.linalg.norm(z - zo) <= 1e-12 * np.linalg.norm(zo), k


@pytest.mark.parametrize("name", ["grid3d_48", "grid2d_256"])
def test_serial_segment_path_is_bit_exact(eng, name, monkeypatch):
    """The optional serial-segment launch (tiny trailing levels solved by one
    block through shared memory) gives the same bytes as the dataflow path."""
    A, F = problem(name)
    O = oracle.Oracle(A, F)
    monkeypatch.setenv("APXB_SEG_LEVEL_ROWS", "64")
    D = native.DeviceFactor(eng, F)
    D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    monkeypatch.delenv("APXB_SEG_LEVEL_ROWS")
    D64_plain = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    x = np.random.default_rng(6).standard_normal(F.m)
    assert np.array_equal(_pair_dev(eng, D, x), O.pair(x))
    z32 = _pair_dev(eng, D32, x)
    want = O.pair(x)
    assert np.linalg.norm(z32 - want) / np.linalg.norm(want) < FP32_SWEEP_RTOL


RZ_RTOL = 1e-12   # r.z: the same products, summed in another (fixed) association than the reference's


@pytest.mark.parametrize("name", gc.NAMES)
def test_apply_fused_and_rz_match_reference_golden(eng, name):
    """apxb_apply on a fresh factor is the reference's first apply_fused of a
    solve (preconditioner.h:370-377): z, and r.z returned beside it."""
    A, F, g = gc.case(name)
    D = native.DeviceFactor(eng, F)
    z, rz = D.apply(g["b"])
    zf, rz_ref = g["apply_fused"], float(g["rz"])
    if F.sddm:
        assert np.array_equal(z, zf)
    else:
        assert np.linalg.norm(z - zf) <= 1e-12 * np.linalg.norm(zf)
    assert abs(rz - rz_ref) <= RZ_RTOL * abs(rz_ref), (rz, rz_ref)
    assert abs(rz - float(np.dot(g["b"], z))) <= RZ_RTOL * abs(rz)


def test_apply_rz_over_the_center_k_schedule(eng):
    """r.z of every application of a 12-application schedule (the 10th centres)
    against the oracle's apply_fused with the same r_sum."""
    A, F, g = gc.case("grid2d_32")
    D = native.DeviceFactor(eng, F)
    O = oracle.Oracle(A, F)
    b = g["b"]
    for k in range(12):
        z, rz = D.apply(b)
        zo, rzo = O.apply_fused(b, float(b.sum()), reset=(k == 0))
        assert np.linalg.norm(z - zo) <= 1e-12 * np.linalg.norm(zo), k
        assert abs(rz - rzo) <= RZ_RTOL * abs(rzo), (k, rz, rzo)
