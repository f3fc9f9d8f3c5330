"""Host logic of the product, no GPU: the C ABI loads and exports every
symbol of include/apxb200.h, and its factor preparation (drop, transpose,
levels, sum modes) is byte-identical to the reference's SpTRSV setup."""
import ctypes

import numpy as np
import pytest

from apxchol_b200 import native, refsetup
from tests import golden_cases as gc
from tests.problems import problem

import oracle


def test_library_exports_every_header_symbol():
    lib = native.load()
    syms = native.header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert b"sm_100a" in lib.apxb_version()


@pytest.mark.parametrize("name", gc.NAMES)
def test_prepare_matches_reference_golden(name):
    A, F, g = gc.case(name)
    hp = native.prepare_host(F)
    for k in ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx", "csc_val"):
        assert np.array_equal(hp[k], g[k]), k


@pytest.mark.parametrize("name", ["grid2d_256", "grid3d_48", "regular_3000", "rmat_12", "path_200"])
def test_prepare_matches_oracle(name):
    A, F = problem(name)
    hp = native.prepare_host(F)
    op = oracle.prepare(F)
    for k in ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx", "csc_val", "fwd_thin", "bck_thin"):
        assert np.array_equal(hp[k], op[k]), k
    assert hp["levels"] == (op["n_fwd_levels"], op["n_bck_levels"])


def test_prepare_without_rounds_uses_topological_levels():
    A, F = problem("grid2d_64")
    F2 = refsetup.Factor(n=F.n, colptr=F.colptr, rowidx=F.rowidx, vals=F.vals, perm=F.perm, sddm=F.sddm,
                         rounds=np.zeros(0, np.uint64))
    hp = native.prepare_host(F2)
    op = oracle.prepare(F2)
    assert np.array_equal(hp["fwd_thin"], op["fwd_thin"]) and np.array_equal(hp["bck_thin"], op["bck_thin"])
    assert hp["levels"] == (op["n_fwd_levels"], op["n_bck_levels"])


def test_prepare_drop_off_keeps_every_entry():
    A, F = problem("grid3d_24")
    hp = native.prepare_host(F, drop_rel=0.0)
    assert hp["nnz"] == F.nnz           # SDDM: L11 is the whole factor


def _broken(F, how):
    colptr, rowidx, vals, perm = F.colptr.copy(), F.rowidx.copy(), F.vals.copy(), F.perm.copy()
    if how == "diag":
        rowidx[colptr[3]], rowidx[colptr[3] + 1] = rowidx[colptr[3] + 1], rowidx[colptr[3]]
    elif how == "perm":
        perm[0] = perm[1]
    elif how == "negdiag":
        vals[colptr[5]] = -1.0
    elif how == "range":
        rowidx[colptr[F.n] - 1] = F.n + 7
    return refsetup.Factor(n=F.n, colptr=colptr, rowidx=rowidx, vals=vals, perm=perm, sddm=F.sddm, rounds=F.rounds)


@pytest.mark.parametrize("how", ["diag", "perm", "negdiag", "range"])
def test_malformed_factor_is_rejected(how):
    A, F = problem("grid2d_64")
    with pytest.raises(native.ApxbError) as ei:
        native.prepare_host(_broken(F, how))
    assert ei.value.code == native.ERR_BAD_FACTOR


def test_factorization_is_deterministic_for_fixed_threads():
    from apxchol_b200 import gen
    A = gen.grid3d(16, seed=1)
    F1 = refsetup.factorize(A, seed=0, threads=4)
    F2 = refsetup.factorize(A, seed=0, threads=4)
    for k in ("colptr", "rowidx", "vals", "perm", "rounds"):
        assert np.array_equal(getattr(F1, k), getattr(F2, k)), k


@pytest.mark.parametrize("name", ["grid3d_24", "rmat_12", "path_200"])
def test_threaded_preparation_matches_serial(name, monkeypatch):
    """The threaded host preparation (the L11 drop, the CSR transpose, the
    plans' fills) gives the same arrays as the serial passes, whatever the
    thread count, including more threads than columns."""
    A, F = problem(name)
    outs = []
    for t in ("1", "3", "8", "64"):
        monkeypatch.setenv("APXB_PREP_THREADS", t)
        outs.append((native.prepare_host(F), native.batch_plan_host(F, 16)))
    base, plans = outs[0]
    for o, pl in outs[1:]:
        assert pl == plans
        for key, v in base.items():
            assert np.array_equal(o[key], v) if isinstance(v, np.ndarray) else o[key] == v, key


@pytest.mark.parametrize("name", ["grid2d_64", "grid3d_24", "rmat_12", "regular_3000", "path_200"])
@pytest.mark.parametrize("k", [1, 4, 8, 16, 32, 64, 128])
def test_batch_plans_hold_their_invariants(name, k):
    """The batch sweep plans (column lanes, oldest-dependency-first entries,
    chunked claims) pass the same checks apxb_batch_create runs: every row once, items within one level in level order, every
    dependency in an older level, diagonals last, chunks covering the items."""
    A, F = problem(name)
    (fi, bi), (fc, bc) = native.batch_plan_host(F, k)
    rows_per_item_max = 32 // (k // 4 if k >= 8 else 1)
    m = F.n if F.sddm else F.n - 1
    for items, chunks in ((fi, fc), (bi, bc)):
        assert m / rows_per_item_max <= items <= m
        assert 1 <= chunks <= items


def test_factor_file_round_trip(tmp_path):
    """A saved factor loads back field for field and prepares to the same arrays."""
    from apxchol_b200.factor_io import load_factor, save_factor
    A, F = problem("grid3d_24")
    save_factor(tmp_path / "f.npz", F)
    G = load_factor(tmp_path / "f.npz")
    assert G.n == F.n and G.sddm == F.sddm and G.lumped == F.lumped
    for name in ("colptr", "rowidx", "vals", "perm", "rounds"):
        assert np.array_equal(getattr(G, name), getattr(F, name)), name
    a, b = native.prepare_host(F), native.prepare_host(G)
    for key in ("csr_ptr", "csr_idx", "csr_val", "csc_val"):
        assert np.array_equal(a[key], b[key])
    np.savez(tmp_path / "bad.npz", format=np.array("something else"))
    with pytest.raises(ValueError):
        load_factor(tmp_path / "bad.npz")


_OOM_CHILD = r"""
import resource, sys
sys.path.insert(0, sys.argv[1])
from apxchol_b200 import native
from tests.problems import problem
A, F = problem("grid3d_48")
native.load()
vm = int([l for l in open("/proc/self/status") if l.startswith("VmSize")][0].split()[1]) * 1024
lim = vm + int(sys.argv[2]) * 2**20
resource.setrlimit(resource.RLIMIT_AS, (lim, lim))
try:
    native.prepare_host(F)
    print("ok")
except Exception as e:
    print("error:", e)
"""


@pytest.mark.parametrize("extra_mb", [4, 16])
def test_host_allocation_failure_is_a_status(extra_mb):
    """A host allocation that fails inside the threaded preparation (the
    address space capped just above the process's current use, 8 threads
    forced) comes back as an error status with its message; the process
    survives. A thread that cannot start leaves its share to the caller."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, APXB_PREP_THREADS="8")
    r = subprocess.run([sys.executable, "-c", _OOM_CHILD, root, str(extra_mb)], capture_output=True, text=True,
                       env=env, cwd=root, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "host allocation failed" in r.stdout, (r.stdout, r.stderr[-2000:])


def test_abi_rejects_bad_arguments_without_a_gpu():
    """Every entry point given NULL handles or out-of-range arguments returns
    APXB_ERR_INVALID with a message, before touching the device (the
    reference throws std::runtime_error for the same misuse, cuda.h:36-39)."""
    lib = native.load()
    info = native.FactorInfo()
    calls = {
        "apxb_factor_info_get": (None, ctypes.byref(info)),
        "apxb_sweep": (None, None, 0, None, None),
        "apxb_sweep_pair": (None, None, None, None),
        "apxb_sweep_pair_multi": (None, None, 4, None, None),
        "apxb_sweep_pair_host": (None, None, None, None),
        "apxb_apply": (None, None, None, None, 0, None),
        "apxb_pcg": (None, None, None, None, None, 1e-8, 10, 0, 0, None),
        "apxb_batch_admit": (None, 0, None, 1e-8, 10, 0),
        "apxb_batch_step": (None, 1, None),
        "apxb_batch_retire": (None, 0, None, 0),
        "apxb_batch_set_refresh": (None, 25),
    }
    for name, args in calls.items():
        rc = getattr(lib, name)(*args)
        assert rc == native.ERR_INVALID, (name, rc)
        assert lib.apxb_last_error(), name
    A, F = problem("path_200")
    items, chunks = np.zeros(2, np.uint32), np.zeros(2, np.uint32)
    cp_, ri = np.ascontiguousarray(F.colptr, np.uint32), np.ascontiguousarray(F.rowidx, np.uint32)
    va, pe = np.ascontiguousarray(F.vals, np.float32), np.ascontiguousarray(F.perm, np.uint32)
    rc = lib.apxb_batch_plan_host(F.n, native.ptr(cp_), native.ptr(ri), native.ptr(va), native.ptr(pe), int(F.sddm),
                                  None, 0, -1.0, 3, native.ptr(items), native.ptr(chunks))
    assert rc == native.ERR_INVALID and b"k must be" in lib.apxb_last_error()
