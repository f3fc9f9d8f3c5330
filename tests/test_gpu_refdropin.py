"""The reference's own solve phase on apxb200's kernels (gpu).

tests/cpp/refdropin builds the apxchol reference's unmodified src/solve.cpp
and preconditioner.h with APXCHOL_USE_CUDA against the replacement headers in
include/apxchol_compat (cuda_sptrsv, cuda_pcg, cuda_ctx over libapxb200). Its
call sites then run on the sm_100a kernels:
  * apxchol::solve (src/solve.cpp:681-737): the reference factorizes, then
    the replacement cuda_pcg runs the whole loop on the device;
  * cpu_solver::apply / cpu_solver::solve on a given factor: every
    preconditioner application goes through apx_cholesky::trsv_, the
    replacement cuda_sptrsv (host-pointer pair solves).
Checked against the reference's CPU build (oracle/_ref) on the same factor:
iterations within +-2, solutions within the PCG tolerance, applications
within 1e-12 relative. (The GPU class receives no elimination rounds from
preconditioner.h, so its sweep levels are the dependency levels and the sum
order of some rows differs from the CPU build's: equal to roundoff, not bit
for bit.)
"""
import ctypes
import os

import numpy as np
import pytest

from apxchol_b200 import gen, refsetup
from tests.problems import SPECS, problem

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tests", "cpp", "refdropin", "_ref", "libapxdropin.so")
TOL = 1e-8
TRUE_RES_FACTOR = 10.0
APPLY_RTOL = 1e-12

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(LIB) and oracle.ref_available()),
                                 reason="drop-in build (tests/cpp/refdropin/_ref) or oracle/_ref absent")]

c_p = ctypes.c_void_p


def _p(a):
    return a.ctypes.data


@pytest.fixture(scope="module")
def lib():
    import torch
    torch.cuda.init()
    L = ctypes.CDLL(LIB)
    L.dap_last_error.restype = ctypes.c_char_p
    L.dap_set_threads.argtypes = [ctypes.c_int]
    L.dap_solve.argtypes = [ctypes.c_int, c_p, c_p, c_p, c_p, ctypes.c_double, ctypes.c_int, ctypes.c_uint,
                            c_p, c_p, c_p, c_p]
    L.dap_solver_create.argtypes = [ctypes.c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_p, ctypes.c_int, c_p,
                                    ctypes.c_uint32, ctypes.POINTER(c_p)]
    L.dap_solver_free.argtypes = [c_p]
    L.dap_apply.argtypes = [c_p, c_p, c_p, ctypes.c_int]
    L.dap_solver_solve.argtypes = [c_p, c_p, c_p, ctypes.c_double, ctypes.c_int, c_p, c_p]
    L.dap_trsv_info.argtypes = [c_p] + [c_p] * 5
    L.dap_set_threads(refsetup.DEFAULT_THREADS)   # the thread count the test factors are pinned to
    return L


def _check(L, rc):
    if rc != 0:
        raise RuntimeError(L.dap_last_error().decode())


def _true_res(A, b, x):
    return float(np.linalg.norm(b - A.matvec(x)) / np.linalg.norm(b))


@pytest.mark.parametrize("name", ["grid3d_24", "grid2d_64", "regular_3000", "rmat_12"])
def test_apxchol_solve_runs_on_the_new_kernels(lib, name):
    """apxchol::solve: factorization by the reference (seed and threads as the
    test factor), GPU-resident PCG by the replacement cuda_pcg."""
    A, F = problem(name)
    seed = SPECS[name][1]
    b = gen.rhs(A.n, 77, not F.sddm)
    cp_ = np.ascontiguousarray(A.colptr, np.int32)
    ri = np.ascontiguousarray(A.rowidx, np.int32)
    va = np.ascontiguousarray(A.vals, np.float64)
    x = np.empty(A.n)
    it = ctypes.c_int()
    res = ctypes.c_double()
    vram = ctypes.c_double()
    _check(lib, lib.dap_solve(A.n, _p(cp_), _p(ri), _p(va), _p(b), TOL, 500, seed, _p(x), ctypes.byref(it),
                              ctypes.byref(res), ctypes.byref(vram)))
    oracle.set_threads(refsetup.DEFAULT_THREADS)
    xr, itr, _, _ = oracle.Ref(A, F).solve(b, TOL, 500)
    assert abs(it.value - itr) <= 2, (it.value, itr)
    assert res.value < TOL
    assert _true_res(A, b, x) < TRUE_RES_FACTOR * TOL
    assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
    assert vram.value > 0.0      # the reference's cudaMemGetInfo sample saw the solve's device memory


@pytest.fixture
def solver(lib, request):
    A, F = problem(request.param)
    keep = [np.ascontiguousarray(a) for a in (A.colptr, A.rowidx, A.vals)] + \
           [np.ascontiguousarray(F.colptr, np.uint32), np.ascontiguousarray(F.rowidx, np.uint32),
            np.ascontiguousarray(F.vals, np.float32), np.ascontiguousarray(F.perm, np.uint32),
            np.ascontiguousarray(F.rounds, np.uint64)]
    h = c_p()
    _check(lib, lib.dap_solver_create(A.n, *[_p(k) for k in keep[:7]], int(F.sddm),
                                      _p(keep[7]) if keep[7].size else None, keep[7].size, ctypes.byref(h)))
    yield A, F, h
    lib.dap_solver_free(h)


@pytest.mark.parametrize("solver", ["grid2d_64", "grid3d_24"], indirect=True)
def test_cpu_solver_apply_and_solve_through_the_gpu_sptrsv(lib, solver):
    A, F, h = solver
    oracle.set_threads(refsetup.DEFAULT_THREADS)
    R = oracle.Ref(A, F)
    st, dr, dev = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    grid, fp16 = ctypes.c_int(), ctypes.c_int()
    _check(lib, lib.dap_trsv_info(h, ctypes.byref(st), ctypes.byref(dr), ctypes.byref(grid), ctypes.byref(dev),
                                  ctypes.byref(fp16)))
    assert st.value == R.nnz_stored and grid.value > 0 and dev.value > 0 and fp16.value == 0
    b = gen.rhs(A.n, 5, not F.sddm)
    for k in range(12):                  # the center-k schedule: the 10th application centres (Laplacian)
        z = np.empty(A.n)
        _check(lib, lib.dap_apply(h, _p(b), _p(z), int(k == 0)))
        zr = R.apply(b, reset=(k == 0))
        assert np.linalg.norm(z - zr) <= APPLY_RTOL * np.linalg.norm(zr), k
    x = np.empty(A.n)
    it, res = ctypes.c_int(), ctypes.c_double()
    _check(lib, lib.dap_solver_solve(h, _p(b), _p(x), TOL, 500, ctypes.byref(it), ctypes.byref(res)))
    xr, itr, _, _ = R.solve(b, TOL, 500)
    assert abs(it.value - itr) <= 2, (it.value, itr)
    assert np.linalg.norm(x - xr) <= 1e-6 * np.linalg.norm(xr)
