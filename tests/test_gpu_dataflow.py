"""The reference's raw dataflow sweep entry points on apxb200's kernel (gpu).

apxchol::dataflow_solve / dataflow_solve_fp16 (the replacement
cuda_dataflow.h, csrc/tagflow.cu) driven exactly as the reference's GPU test
drives its own kernel (tests/test_sptrsv_drop.cpp:1228-1330): the reference's
cuda_host.h builds the L11 storage (fp32, and fp16 column-scaled), the CSR of
L and of L^T and each direction's batch plan with dataflow_build_plan, at
three segmentation settings -- off, the reference's shipped shape (1024-entry
segments for rows over 2048 off-diagonals) and the torture setting (every row
cut into 256-entry segments). The gates are the reference test's own:
  * every sweep within 1e-6 (max |diff| / max |ref|, kSweepTol) of a serial
    fp64 sweep over the same arrays;
  * bit-identical results on a one-block grid (8 warps against every batch:
    the deadlock torture) and the resident grid, and across repeated launches.
The harness is tests/cpp/refdropin/dataflow_harness.cpp."""
import ctypes
import os

import numpy as np
import pytest

from tests.problems import problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tests", "cpp", "refdropin", "_ref", "libapxdropin.so")
SWEEP_TOL = 1e-6          # kSweepTol, test_sptrsv_drop.cpp:1204
DROP_REL = 1e-4           # the drop the reference test sets (scoped_drop_env("1e-4"))
SEG_CFGS = [(0, 0, 4096), (1024, 2048, 4096), (256, 0, 4096)]

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(LIB), reason="drop-in build (tests/cpp/refdropin/_ref) absent")]

c_p = ctypes.c_void_p


@pytest.fixture(scope="module")
def lib():
    import torch
    torch.cuda.init()
    L = ctypes.CDLL(LIB)
    L.dap_df_last_error.restype = ctypes.c_char_p
    L.dap_df_create.argtypes = [ctypes.c_int, c_p, c_p, c_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, ctypes.POINTER(c_p)]
    L.dap_df_free.argtypes = [c_p]
    L.dap_df_info.argtypes = [c_p, c_p, c_p, c_p, c_p]
    L.dap_df_sweep.argtypes = [c_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, c_p, c_p]
    L.dap_df_serial.argtypes = [c_p, ctypes.c_int, ctypes.c_int, c_p, c_p]
    return L


def _check(L, rc):
    if rc != 0:
        raise RuntimeError(L.dap_df_last_error().decode())


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


class Sweeps:
    def __init__(self, L, name, cfg):
        A, F = problem(name)
        self.L = L
        self.keep = [np.ascontiguousarray(F.colptr, np.uint32), np.ascontiguousarray(F.rowidx, np.uint32),
                     np.ascontiguousarray(F.vals, np.float32)]
        self.h = c_p()
        _check(L, L.dap_df_create(F.n, *[k.ctypes.data for k in self.keep], F.m, *cfg, DROP_REL,
                                  ctypes.byref(self.h)))
        m = ctypes.c_int()
        self.nb, self.split, self.slots = (np.zeros(2, np.int32) for _ in range(3))
        L.dap_df_info(self.h, ctypes.byref(m), self.nb.ctypes.data, self.split.ctypes.data, self.slots.ctypes.data)
        self.m = m.value

    def gpu(self, reverse, fp16, rhs, grid=0):
        rhs = np.ascontiguousarray(rhs, np.float32)
        out = np.empty(self.m, np.float32)
        _check(self.L, self.L.dap_df_sweep(self.h, reverse, fp16, grid, rhs.ctypes.data, out.ctypes.data))
        return out

    def serial(self, reverse, fp16, rhs):
        rhs = np.ascontiguousarray(rhs, np.float32)
        out = np.empty(self.m)
        _check(self.L, self.L.dap_df_serial(self.h, reverse, fp16, rhs.ctypes.data, out.ctypes.data))
        return out

    def close(self):
        self.L.dap_df_free(self.h)


@pytest.mark.parametrize("cfg", SEG_CFGS, ids=["seg_off", "seg_shipped", "seg_torture"])
@pytest.mark.parametrize("name", ["grid3d_24", "rmat_14"])
def test_dataflow_sweeps_match_the_serial_reference(lib, name, cfg):
    S = Sweeps(lib, name, cfg)
    try:
        if cfg[0] == 256:
            assert S.split[0] > 0 and S.split[1] > 0       # the torture setting splits rows both ways
        for fp16 in (0, 1):
            x = np.random.default_rng(21 + fp16).standard_normal(S.m).astype(np.float32)
            y = S.gpu(0, fp16, x)
            assert _rel(y, S.serial(0, fp16, x)) < SWEEP_TOL, (name, cfg, fp16, "forward")
            z = S.gpu(1, fp16, y)
            assert _rel(z, S.serial(1, fp16, y)) < SWEEP_TOL, (name, cfg, fp16, "back")
            # one block (8 warps against every batch), then the resident grid again: same bits
            assert np.array_equal(S.gpu(0, fp16, x, grid=1), y)
            assert np.array_equal(S.gpu(1, fp16, y, grid=1), z)
            assert np.array_equal(S.gpu(0, fp16, x), y)
    finally:
        S.close()


def test_dataflow_hub_rows_are_split_and_segments_change_nothing_unsplit(lib):
    """On the power-law factor (a 3676-entry row), the shipped setting splits
    the hub rows and keeps every other row unsplit; the result stays within the
    gate of the unsplit plan's and of the serial sweep."""
    off = Sweeps(lib, "rmat_14", SEG_CFGS[0])
    on = Sweeps(lib, "rmat_14", SEG_CFGS[1])
    try:
        assert off.split.sum() == 0 and on.split.sum() > 0
        x = np.random.default_rng(5).standard_normal(off.m).astype(np.float32)
        for reverse in (0, 1):
            a, b = off.gpu(reverse, 0, x), on.gpu(reverse, 0, x)
            ref = off.serial(reverse, 0, x)
            assert _rel(a, ref) < SWEEP_TOL and _rel(b, ref) < SWEEP_TOL
    finally:
        off.close()
        on.close()
