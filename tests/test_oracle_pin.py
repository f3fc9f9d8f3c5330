"""The oracle (oracle/apxoracle.c) pinned against the apxchol reference itself:
golden outputs the reference produced (tests/golden) and, where the reference
build is present, the reference run live on larger systems."""
import numpy as np
import pytest

import oracle
from tests import golden_cases as gc
from tests.problems import problem

ARRAYS = ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx", "csc_val")


@pytest.mark.parametrize("name", gc.NAMES)
def test_oracle_reproduces_reference_golden(name):
    A, F, g = gc.case(name)
    O = oracle.Oracle(A, F, nt=1)
    for k in ARRAYS:
        assert np.array_equal(O.p[k], g[k]), k
    y = O.sweep(0, g["x"])
    assert np.array_equal(y, g["fwd"])                      # bit-exact forward sweep
    assert np.array_equal(O.sweep(1, y), g["pair"])         # bit-exact backward sweep
    assert np.array_equal(O.apply(g["b"]), g["apply"])
    zf, rz = O.apply_fused(g["b"], float(g["b"].sum()))
    assert np.array_equal(zf, g["apply_fused"]) and rz == float(g["rz"])
    x, it, res = O.solve(g["b"], 1e-8, 500)
    assert it == int(g["pcg_iters"]) and res == float(g["pcg_res"])
    assert np.array_equal(x, g["pcg_x"])


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("name,nt", [("grid2d_64", 4), ("grid3d_24", 4), ("regular_3000", 3), ("rmat_12", 4),
                                     ("path_200", 2)])
def test_oracle_matches_reference_live(name, nt):
    A, F = problem(name)
    oracle.set_threads(nt)
    R = oracle.Ref(A, F)
    O = oracle.Oracle(A, F, nt=nt)
    ra = R.arrays()
    for k in ARRAYS:
        assert np.array_equal(ra[k], O.p[k]), k
    assert R.fwd_levels == O.p["n_fwd_levels"] and R.bck_levels == O.p["n_bck_levels"]
    assert np.array_equal(np.bincount(O.p["fwd_level"], minlength=R.fwd_levels), R.level_sizes(True))
    assert np.array_equal(np.bincount(O.p["bck_level"], minlength=R.bck_levels), R.level_sizes(False))
    x = np.random.default_rng(1).standard_normal(F.m)
    y = R.forward(x)
    assert np.array_equal(y, O.sweep(0, x))
    assert np.array_equal(R.transpose(y), O.sweep(1, y))
    from apxchol_b200 import gen
    b = gen.rhs(A.n, 3, not F.sddm)
    assert np.array_equal(R.apply(b), O.apply(b))
    z1, rz1 = R.apply_fused(b, b.sum())
    z2, rz2 = O.apply_fused(b, b.sum())
    assert np.array_equal(z1, z2) and rz1 == rz2
    x1, it1, r1, _ = R.solve(b)
    x2, it2, r2 = O.solve(b)
    assert it1 == it2 and r1 == r2 and np.array_equal(x1, x2)


@needs_ref
def test_center_k_schedule_matches_reference():
    """Twelve consecutive Eigen-seam applications: only the 10th centres."""
    A, F = problem("grid2d_64")
    oracle.set_threads(1)
    R = oracle.Ref(A, F)
    O = oracle.Oracle(A, F, nt=1)
    b = np.random.default_rng(5).standard_normal(A.n)
    for k in range(12):
        assert np.array_equal(R.apply(b, reset=(k == 0)), O.apply(b, reset=(k == 0))), k


@pytest.mark.skipif(not (oracle.ref_available() and __import__("os").path.exists(oracle.REF_LIB_V4)
                         and oracle.host_has_avx512()),
                    reason="x86-64-v4 reference build or an AVX-512 host absent")
def test_avx512_reference_build_gives_the_same_bits():
    """The timed CPU baseline may run the x86-64-v4 build of the reference; it
    must be the same arithmetic as the portable build the oracle is pinned to."""
    A, F = problem("grid3d_24")
    b = np.random.default_rng(8).standard_normal(A.n)
    out = []
    for path in (oracle.REF_LIB, oracle.REF_LIB_V4):
        oracle.set_threads(4, path)
        R = oracle.Ref(A, F, lib_path=path)
        y = R.forward(b[:R.m])
        x, it, res, _ = R.solve(b, 1e-8, 500)
        out.append((y, R.transpose(y), x, it, res))
    for a, c in zip(out[0], out[1]):
        assert np.array_equal(a, c)
