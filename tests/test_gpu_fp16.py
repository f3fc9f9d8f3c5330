"""The fp16 factor storage on the GPU (gpu): the fp32 sweeps over binary16
values of the column-scaled factor, a per-row fp32 diagonal and the backward
right-hand side times (1/s)^2 in fp64.

The gates are the reference's own (tests/test_sptrsv_drop.cpp:1198-1206):
- each sweep against a serial fp64 host sweep over the same fp16 arrays
  (oracle.sweep16, after host_reference_sweep :1100-1127):
  max |diff| / max |ref| < 1e-6;
- the pair against the CPU backend's fp64 pair of the fp32-stored factor:
  < 1e-3 (fp16 rounds every off-diagonal to 11 bits, so the pair is a
  slightly different preconditioner);
- bit-identical results at any sweep grid."""
import numpy as np
import pytest

from apxchol_b200 import native
from tests.problems import problem

import oracle

pytestmark = pytest.mark.gpu

SWEEP_TOL = 1e-6      # kSweepTol, test_sptrsv_drop.cpp:1204
PAIR_TOL_FP16 = 1e-3  # kPairTolFp16, test_sptrsv_drop.cpp:1206


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


def _run(eng, fn, x):
    import torch
    dx = _dev(x)
    dz = torch.empty_like(dx)
    torch.cuda.synchronize()
    fn(dx, dz)
    eng.sync()
    return dz.cpu().numpy()


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


@pytest.mark.parametrize("name,rel", [("grid3d_24", -1.0), ("grid3d_24", 0.0), ("grid2d_64", -1.0),
                                      ("rmat_12", -1.0), ("path_200", -1.0)])
def test_fp16_sweeps_match_the_host_sweep(eng, name, rel):
    A, F = problem(name)
    h = native.prepare_host_fp16(F, rel)
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP16, drop_rel=rel)
    assert D.info.precision == native.PREC_FP16 and D.info.nnz_stored == h["nnz"]
    m = h["m"]
    x = np.random.default_rng(11).standard_normal(m)
    y = _run(eng, lambda a, b: D.sweep(0, a, b), x)
    # the kernels narrow their fp64 input to fp32 first: the host sweep gets the same input
    y_ref = oracle.sweep16(0, h, x.astype(np.float32)).astype(np.float32)
    assert _rel(y, y_ref) < SWEEP_TOL
    is2 = h["inv_scale"].astype(np.float64) ** 2
    z = _run(eng, lambda a, b: D.sweep(1, a, b), y)
    z_ref = oracle.sweep16(1, h, y.astype(np.float32), is2).astype(np.float32)
    assert _rel(z, z_ref) < SWEEP_TOL


@pytest.mark.parametrize("name", ["grid3d_24", "grid2d_64", "regular_3000", "rmat_12", "grid3d_48"])
def test_fp16_pair_within_the_reference_gate_and_schedule_free(eng, name):
    A, F = problem(name)
    O = oracle.Oracle(A, F)
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP16)
    x = np.random.default_rng(12).standard_normal(F.m)
    want = O.pair(x)
    got = _run(eng, D.sweep_pair, x)
    assert _rel(got, want) < PAIR_TOL_FP16
    for grid in (1, 7, 0):
        eng.set_sweep_grid(grid)
        assert np.array_equal(_run(eng, D.sweep_pair, x), got), grid
    eng.set_sweep_grid(0)
    assert np.array_equal(D.sweep_pair_host(x), got)


def test_fp16_apply_and_bytes(eng):
    """apx_cholesky::apply with the fp16 factor (Laplacian with centring, and
    SDDM) stays within the pair gate of the reference apply, and the factor
    holds fewer device bytes than the fp32 one (6 instead of 8 per stored
    entry and direction, plus 12 per row)."""
    for name in ("grid2d_64", "grid3d_24"):
        A, F = problem(name)
        O = oracle.Oracle(A, F)
        D16 = native.DeviceFactor(eng, F, precision=native.PREC_FP16)
        D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
        assert D16.info.device_bytes < D32.info.device_bytes
        b = np.random.default_rng(13).standard_normal(F.n)
        if not F.sddm:
            b -= b.mean()
        for k in range(12):                   # the center-k schedule: the 10th application centres
            z, _ = D16.apply(b)
            zo = O.apply(b, reset=(k == 0))
            assert _rel(z, zo) < PAIR_TOL_FP16, (name, k)
        D16.close()
        D32.close()
