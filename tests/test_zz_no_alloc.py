"""apxb_sweep_pair_noalloc (gpu): the fp64 sweep pair for callers that cannot
allocate device memory in the call -- hosts that reserve the GPU's memory for
their own pool, and loops that cannot take the device-wide synchronisation of
cudaMalloc / cudaFree. Its intermediate vectors live in a fixed library-owned
device array (at most 65,536 factor rows), so the call allocates nothing.

Checked against apxb_sweep_pair, the allocating entry point, through the C ABI
on two calls in a row with different inputs (the second call must not see the
first call's leftovers in the shared array). The tolerance is the one the fp64
sweep tests use: none -- both must give the same bits. This file sorts last so
that a stop-at-first-failure run has run every other test before it."""
import numpy as np
import pytest

from apxchol_b200 import native
from tests.problems import problem

pytestmark = pytest.mark.gpu
MAX_ROWS = 65536


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def _noalloc(eng, D, d_in, d_out):
    native.check(eng.lib.apxb_sweep_pair_noalloc(eng.h, D.h, native.ptr(d_in), native.ptr(d_out)))


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_24"])
def test_noalloc_matches_sweep_pair_on_two_calls(eng, name):
    import torch
    A, F = problem(name)
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    try:
        assert D.m <= MAX_ROWS
        rng = np.random.default_rng(11)
        for call in range(2):
            x = torch.from_numpy(rng.standard_normal(D.m)).cuda()
            want = torch.empty_like(x)
            D.sweep_pair(x, want)
            got = torch.full_like(x, float("nan"))
            _noalloc(eng, D, x, got)
            assert np.array_equal(got.cpu().numpy(), want.cpu().numpy()), f"call {call + 1}"
    finally:
        D.close()


def test_noalloc_on_a_fresh_factor_allocates_nothing(eng):
    """The first sweep a factor ever runs goes through the no-alloc entry
    point: the factor's own work vectors do not exist yet, and the call must
    not create them (engine memory and the factor's device bytes unchanged).
    Its result must still be the allocating pair's, bit for bit."""
    import torch
    A, F = problem("grid2d_256")
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    try:
        x = torch.from_numpy(np.random.default_rng(12).standard_normal(D.m)).cuda()
        got = torch.full_like(x, float("nan"))
        torch.cuda.synchronize()
        used0, bytes0 = eng.memory_used(), D.get_info().device_bytes
        _noalloc(eng, D, x, got)
        assert eng.memory_used() == used0
        assert D.get_info().device_bytes == bytes0
        want = torch.empty_like(x)
        D.sweep_pair(x, want)
        assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())
    finally:
        D.close()


def test_noalloc_rejects_what_it_cannot_hold(eng):
    import torch
    A, F = problem("grid3d_48")          # m = 110,592 rows > 65,536
    D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
    try:
        x = torch.zeros(D.m, dtype=torch.float64, device="cuda")
        with pytest.raises(native.ApxbError) as ex:
            _noalloc(eng, D, x, x)
        assert ex.value.code == native.ERR_INVALID and "65536" in str(ex.value)
    finally:
        D.close()
    A, F = problem("grid3d_24")
    D32 = native.DeviceFactor(eng, F, precision=native.PREC_FP32)
    try:
        x = torch.zeros(D32.m, dtype=torch.float64, device="cuda")
        with pytest.raises(native.ApxbError) as ex:
            _noalloc(eng, D32, x, x)
        assert ex.value.code == native.ERR_INVALID and "fp64" in str(ex.value)
    finally:
        D32.close()
