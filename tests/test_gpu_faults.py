"""Failure detection on the GPU without faulting it (gpu): a sweep wait that
can never be satisfied ends with APXB_ERR_TIMEOUT after its budget and the
engine stays usable; the device-memory budget refuses an allocation."""
import numpy as np
import pytest

from apxchol_b200 import native
from tests.problems import problem

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def test_stalled_wait_times_out_and_engine_recovers(eng):
    A, F = problem("grid2d_64")
    D = native.DeviceFactor(eng, F)
    hp = D.arrays()
    # rows >= 32 that read a row < 32 in the forward sweep: they can never be served
    deps = hp["csr_idx"][hp["csr_ptr"][32]:]
    assert (deps < 32).any()
    with pytest.raises(native.ApxbError) as ei:
        eng.lib  # noqa: B018
        native.check(eng.lib.apxb_test_stalled_sweep(eng.h, D.h, 20_000_000))   # 20 ms budget
    assert ei.value.code == native.ERR_TIMEOUT
    # the context is intact: a normal pair still matches the oracle bytes
    O = oracle.Oracle(A, F)
    x = np.random.default_rng(0).standard_normal(F.m)
    assert np.array_equal(D.sweep_pair_host(x), O.pair(x))


def test_memory_budget_refuses_allocation():
    A, F = problem("grid3d_24")
    e = native.Engine(0)
    try:
        e.set_memory_budget(1 << 16)
        with pytest.raises(native.ApxbError) as ei:
            native.DeviceFactor(e, F)
        assert ei.value.code == native.ERR_BUDGET
        e.set_memory_budget(0)
        D = native.DeviceFactor(e, F)
        assert e.memory_used() >= D.info.device_bytes
    finally:
        e.close()
