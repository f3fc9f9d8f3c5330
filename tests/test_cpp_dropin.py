"""The C++ drop-ins (include/apxb200.hpp) driven like the reference's call
sites drive cuda_sptrsv and cuda_pcg: compiled with the host compiler against
the C ABI library, fed a system through a file, and compared bit for bit with
the same calls made through the Python binding."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from apxchol_b200 import gen, native
from tests.problems import problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.dirname(native.LIB_PATH)


def _cxx():
    for c in ("/usr/bin/g++", shutil.which("g++"), shutil.which("c++")):
        if c and os.path.exists(c):
            return c
    pytest.skip("no C++ compiler")


@pytest.fixture(scope="module")
def dropin(tmp_path_factory):
    if not os.path.exists(native.LIB_PATH):
        pytest.skip("library not built")
    exe = str(tmp_path_factory.mktemp("cpp") / "dropin")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin.cpp"), "-L", LIBDIR, "-lapxb200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _write_input(path, A, F, b, y):
    m = F.n if F.sddm else F.n - 1
    with open(path, "wb") as f:
        for arr in (np.array([F.n, m, int(F.sddm)], np.uint32), np.array([F.nnz], np.uint64),
                    np.asarray(F.colptr, np.uint32), np.asarray(F.rowidx, np.uint32),
                    np.asarray(F.vals, np.float32), np.asarray(F.perm, np.uint32),
                    np.array([len(F.rounds)], np.uint32), np.asarray(F.rounds, np.uint64),
                    np.array([A.nnz], np.uint64), np.asarray(A.colptr, np.int32), np.asarray(A.rowidx, np.int32),
                    np.asarray(A.vals, np.float64), np.asarray(b, np.float64), np.asarray(y, np.float64)):
            f.write(np.ascontiguousarray(arr).tobytes())
    return m


def test_dropin_reports_errors_as_exceptions(dropin, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU error path")
    A, F = problem("grid2d_64")
    _write_input(tmp_path / "in.bin", A, F, gen.rhs(A.n, 1, True), np.ones(A.n - 1))
    r = subprocess.run([dropin, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 2, r
    assert r.stderr.startswith("apxb_engine_create:"), r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["grid2d_64", "grid3d_24"])
def test_dropin_matches_the_c_abi(dropin, tmp_path, name):
    A, F = problem(name)
    b = gen.rhs(A.n, 3, not F.sddm)
    m = F.n if F.sddm else F.n - 1
    y = np.random.default_rng(4).standard_normal(m)
    _write_input(tmp_path / "in.bin", A, F, b, y)
    r = subprocess.run([dropin, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = open(tmp_path / "out.bin", "rb").read()
    sweep = np.frombuffer(raw[:8 * m], np.float64)
    x = np.frombuffer(raw[8 * m: 8 * (m + A.n)], np.float64)
    iters = int(np.frombuffer(raw[8 * (m + A.n): 8 * (m + A.n) + 4], np.int32)[0])
    eng = native.Engine(0)
    try:
        D = native.DeviceFactor(eng, F, precision=native.PREC_FP64)
        Op = native.DeviceOperator(eng, A, F.perm)
        assert np.array_equal(sweep, D.sweep_pair_host(y))
        x_ref, res = native.pcg(eng, D, Op, b, tol=1e-8, max_iter=500)
        assert iters == res.iterations
        assert np.array_equal(x, x_ref)
        Op.close(); D.close()
    finally:
        eng.close()


@pytest.mark.parametrize("env,want", [(None, "-1 0 0"), ("1", "1 1 2"), ("0", "0 0 0"), ("yes", "-1 0 0")])
def test_dropin_fp16_switch(tmp_path, env, want):
    """APXCHOL_SPTRSV_FP16=1 selects the fp16 storage (APXB_PREC_FP16 = 2),
    =0 or anything else keeps the default, the bit-exact fp64 sweeps (0)."""
    exe = str(tmp_path / "fp16_env")
    subprocess.run([_cxx(), "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "fp16_env.cpp"), "-L", LIBDIR, "-lapxb200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    e = dict(os.environ)
    e.pop("APXCHOL_SPTRSV_FP16", None)
    if env is not None:
        e["APXCHOL_SPTRSV_FP16"] = env
    r = subprocess.run([exe], capture_output=True, text=True, env=e, check=True)
    assert r.stdout.strip() == want


REFDROPIN = os.path.join(ROOT, "tests", "cpp", "refdropin", "_ref", "libapxdropin.so")


@pytest.mark.skipif(not os.path.exists(REFDROPIN), reason="drop-in build of the reference absent")
def test_reference_dropin_library_resolves_every_symbol():
    """The reference's solve phase compiled against include/apxchol_compat
    (tests/cpp/refdropin) loads with every symbol bound (no GPU needed):
    nothing it calls is left undefined by the replacement headers."""
    import ctypes
    lib = ctypes.CDLL(REFDROPIN, mode=os.RTLD_NOW)
    for name in ("dap_solve", "dap_solver_create", "dap_apply", "dap_solver_solve", "dap_trsv_info"):
        assert hasattr(lib, name), name
