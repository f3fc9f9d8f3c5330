"""The fp16 factor storage (APXB_PREC_FP16) on the host, no GPU.

What an fp16 factor uploads must be, bit for bit, what the reference GPU
backend's own host code builds with APXCHOL_SPTRSV_FP16=1 (cuda_host.h:120-258:
the drop with the fp16 keep predicate, the per-column binary16 narrowing, the
fp32 diagonal with the column's rounding residual, 1/s_j, and the transpose
carrying the same 16-bit patterns), run here from the reference sources
(oracle/_ref). The reference's counterpart is GpuHostPrep.* in
tests/test_sptrsv_drop.cpp:632-720."""
import types

import numpy as np
import pytest

from apxchol_b200 import native
from tests.problems import problem

import oracle

KEYS = ("csc_ptr", "csc_idx", "csc_val16", "csr_ptr", "csr_idx", "csr_val16", "diag", "inv_scale")

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")


def _same(ours, ref):
    for k in KEYS:
        a, b = ours[k], ref[k]
        assert a.shape == b.shape, k
        if a.dtype.kind == "f":
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
        else:
            assert np.array_equal(a.astype(np.int64), b.astype(np.int64)), k
    assert np.array_equal(ours["stats"], ref["stats"])


def _wide_factor(n, seed, sddm):
    """A random lower-triangular factor in the storage contract (columns start
    with a positive diagonal, rows ascending) whose off-diagonals span
    10^-12 .. 1, so the narrowing meets normal, subnormal and flushed
    binary16 values and every rounding case."""
    rng = np.random.default_rng(seed)
    colptr, rowidx, vals = [0], [], []
    for j in range(n):
        below = np.arange(j + 1, n)
        k = min(len(below), int(rng.integers(0, 9)))
        rows = np.sort(rng.choice(below, size=k, replace=False)) if k else np.zeros(0, np.int64)
        rowidx.append(j)
        vals.append(1.0 + rng.random())
        for r in rows:
            rowidx.append(int(r))
            vals.append(-(10.0 ** rng.uniform(-12, 0)) * rng.random())
        colptr.append(len(rowidx))
    return types.SimpleNamespace(n=n, sddm=sddm, colptr=np.array(colptr, np.uint32),
                                 rowidx=np.array(rowidx, np.uint32), vals=np.array(vals, np.float32),
                                 perm=np.arange(n, dtype=np.uint32), rounds=np.zeros(0, np.uint64))


@needs_ref
@pytest.mark.parametrize("name", ["path_200", "grid2d_64", "grid3d_24", "rmat_12", "regular_3000"])
@pytest.mark.parametrize("rel", [-1.0, 0.0, 1e-30])
def test_fp16_storage_is_the_reference_storage(name, rel):
    A, F = problem(name)
    _same(native.prepare_host_fp16(F, rel), oracle.fp16_prep(F, rel))


@needs_ref
@pytest.mark.parametrize("sddm", [True, False])
@pytest.mark.parametrize("rel", [-1.0, 0.0, 1e-30, 1e-3])
def test_fp16_storage_wide_magnitudes(sddm, rel):
    F = _wide_factor(3000, 7 + int(sddm), sddm)
    ours = native.prepare_host_fp16(F, rel)
    _same(ours, oracle.fp16_prep(F, rel))
    if rel == 0.0:
        assert ours["stats"][2] > 0          # teeth: some stored values are flushed
    if rel == 1e-30:
        assert ours["stats"][1] > 0          # the fp16 keep clause drops what fp16 flushes


@needs_ref
@pytest.mark.parametrize("rel", [-1.0, 0.0])
def test_fp16_scale_fallback(rel):
    """Columns whose off-diagonals are ~1e-39 (fp32 subnormals): 1/s overflows
    fp32, so s falls back to 1 (cuda.h:287-301) and their off-diagonals flush
    to zero, folded into the diagonal."""
    F = _wide_factor(2000, 21, True)
    tiny = np.array([1e-39, 5e-40, 1e-40], np.float32)   # 1/s >= 1e39 overflows fp32
    hit = []
    for j in range(0, 1900, 37):
        lo, hi = int(F.colptr[j]), int(F.colptr[j + 1])
        if hi - lo > 1:
            F.vals[lo + 1:hi] = -tiny[np.arange(hi - lo - 1) % 3]
            hit.append(j)
    ours = native.prepare_host_fp16(F, rel)
    _same(ours, oracle.fp16_prep(F, rel))
    assert len(hit) > 10
    assert all(ours["inv_scale"][j] == 1.0 for j in hit)


def test_fp16_values_and_folded_diagonal():
    """Self-checks of the contract without the reference: each stored
    off-diagonal is binary16(v / s) of the fp32 column (numpy's IEEE
    conversion), and the diagonal plus the widened off-diagonals sum to the
    fp32 column / s up to fp32 rounding of the diagonal."""
    A, F = problem("grid3d_24")
    h = native.prepare_host_fp16(F, 0.0)
    p = native.prepare_host(F, 0.0)                      # the same drop (none): the fp32 values
    assert np.array_equal(h["csc_idx"], p["csc_idx"])
    ptr, idx, v32 = p["csc_ptr"], p["csc_idx"], p["csc_val"]
    w = h["csc_val16"].view(np.float16)
    for j in range(0, F.n, 97):
        lo, hi = int(ptr[j]), int(ptr[j + 1])
        off = np.arange(lo + 1, hi)                      # the column starts with its diagonal
        smax = np.max(np.abs(v32[off])) if off.size else np.float32(1.0)
        assert np.float32(1.0) / smax == h["inv_scale"][j]
        q = (v32[off] / smax).astype(np.float16)
        q[np.abs(q.astype(np.float32)) < np.float32(2.0 ** -14)] = 0.0   # subnormals are flushed
        assert np.array_equal(np.abs(w[off].astype(np.float32)), np.abs(q.astype(np.float32))), j
        col = float(v32[lo]) / float(smax) + float(np.sum(v32[off].astype(np.float64) / float(smax)))
        got = float(h["diag"][j]) + float(np.sum(w[off].astype(np.float64)))
        assert abs(got - col) <= 1e-6 * max(1.0, abs(col)), j


@pytest.mark.parametrize("name", ["grid3d_24", "rmat_12", "grid2d_64"])
def test_fp16_storage_applies_the_preconditioner(name):
    """The stored, column-scaled factor applies (L L^T)^-1: the forward sweep
    on L~ = L D^-1, the input of the backward sweep times D^-2, the backward
    sweep on L~^T. In fp64 on the host (oracle.sweep16) this is within the
    reference's fp16 pair gate (1e-3, test_sptrsv_drop.cpp:1206) of the fp64
    pair; measured at most 2e-4."""
    A, F = problem(name)
    h = native.prepare_host_fp16(F)
    m = h["m"]
    x = np.random.default_rng(5).standard_normal(m)
    y = oracle.sweep16(0, h, x)
    z = oracle.sweep16(1, h, y, h["inv_scale"].astype(np.float64) ** 2)
    want = oracle.Oracle(A, F).pair(x)
    assert np.max(np.abs(z - want)) / np.max(np.abs(want)) < 1e-3
