"""Factor preparation on the device (gpu): apxb_factor_create builds the
L11 drop, the CSC -> CSR transpose, the levels, both sweep plans, the batch
plans and the operator's P A P^T with kernels. Every array must be the host
preparation's (host_prep.cpp, pinned to the reference by the CPU tests), byte
for byte: apxb_test_prep_compare builds both and compares them."""
import numpy as np
import pytest

from apxchol_b200 import native, workloads
from tests import golden_cases as gc
from tests.problems import problem

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    import torch
    torch.cuda.init()
    e = native.Engine(0)
    yield e
    e.close()


def _compare(eng, A, F, k, drop_rel=-1.0):
    keep = [np.ascontiguousarray(F.colptr, np.uint32), np.ascontiguousarray(F.rowidx, np.uint32),
            np.ascontiguousarray(F.vals, np.float32), np.ascontiguousarray(F.perm, np.uint32),
            np.ascontiguousarray(F.rounds, np.uint64)]
    ops = [np.ascontiguousarray(A.colptr, np.int32), np.ascontiguousarray(A.rowidx, np.int32),
           np.ascontiguousarray(A.vals, np.float64)] if A is not None else [None] * 3
    native.check(eng.lib.apxb_test_prep_compare(
        eng.h, F.n, *[native.ptr(a) for a in keep[:4]], int(F.sddm), native.ptr(keep[4]), keep[4].size, drop_rel, k,
        *[native.ptr(a) if a is not None else None for a in ops]))


@pytest.mark.parametrize("name", gc.NAMES)
def test_golden_factors(eng, name):
    A, F, _ = gc.case(name)
    for k in (0, 1, 16):
        _compare(eng, A, F, k)


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_48", "regular_3000", "rmat_12", "rmat_14", "path_200"])
@pytest.mark.parametrize("k", [2, 8, 16])
def test_problems(eng, name, k):
    """rmat_14 has factor rows and operator rows longer than 32 entries (the
    block-wide sorts); grid3d_48's high-contrast weights make the drop act."""
    A, F = problem(name)
    _compare(eng, A, F, k)


@pytest.mark.parametrize("drop_rel", [0.0, 1e-2])
def test_drop_settings(eng, drop_rel):
    A, F = problem("grid3d_48")
    _compare(eng, A, F, 16, drop_rel)


def test_bad_factors_fail_alike(eng):
    """Both preparations reject malformed input with the same message."""
    A, F = problem("grid2d_64")
    bad = F.rowidx.copy()
    bad[F.colptr[5]] = 7            # column 5 does not start with its diagonal
    G = type(F)(n=F.n, colptr=F.colptr, rowidx=bad, vals=F.vals, perm=F.perm, sddm=F.sddm, rounds=F.rounds)
    _compare(eng, None, G, 4)
    perm = F.perm.copy()
    perm[0] = perm[1]               # not a permutation
    G = type(F)(n=F.n, colptr=F.colptr, rowidx=F.rowidx, vals=F.vals, perm=perm, sddm=F.sddm, rounds=F.rounds)
    _compare(eng, None, G, 4)


def test_grid128_admission_arrays(eng):
    """The 128^3 benchmark factor (16.3M stored entries) and its operator."""
    A, F = workloads.grid3d_128()
    _compare(eng, A, F, 16)
