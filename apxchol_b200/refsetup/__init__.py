"""The reference's own seeded factorization, loaded from _ref/libapxsetup.so.

The solve phase consumes a factor made by apxchol's unchanged setup phase
(`apxchol::factorize`, src/factorization.cpp:125-175 with the default
`block_greedy` partitioner and `vec_pool` storage). This module builds it
from the reference sources once (Makefile beside this file) and exposes
`factorize(matrix, seed, threads)` returning a `Factor`.

The factor is bit-identical for a fixed (matrix, seed, thread count), so the
thread count is an explicit argument.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libapxsetup.so")
_lib = None

# Thread count the factors of tests and benchmarks are pinned to.
DEFAULT_THREADS = 8


@dataclass
class Factor:
    """apxchol::factorization (include/apxchol/solver/factorization.h:22-56):
    lower-triangular CSC factor with the diagonal first in each column and
    rows ascending, the elimination permutation perm[original] = position,
    the SDDM flag and the per-round independent-set sizes."""
    n: int
    colptr: np.ndarray   # uint32[n+1]
    rowidx: np.ndarray   # uint32[nnz]
    vals: np.ndarray     # float32[nnz]
    perm: np.ndarray     # uint32[n]
    sddm: bool
    rounds: np.ndarray   # uint64[n_rounds]
    lumped: int = 0

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    @property
    def m(self) -> int:
        """Factor dimension the sweeps use: n (SDDM) or n-1 (Laplacian)."""
        return self.n if self.sddm else self.n - 1


def build(ref_root: str | None = None) -> None:
    """Compile the library from the reference sources (ref_root, else
    $APXCHOL_REF: the reference source tree)."""
    import subprocess
    ref_root = ref_root or os.environ.get("APXCHOL_REF", "")
    if not ref_root or not os.path.isdir(ref_root):
        raise RuntimeError("reference source tree not found: pass ref_root or set APXCHOL_REF")
    subprocess.check_call(["make", "-s", "-C", _HERE, f"REF={ref_root}"])


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise RuntimeError(f"reference factorization library missing: {_LIB_PATH} "
                           "(run apxchol_b200.refsetup.build() where the reference tree exists)")
    lib = ctypes.CDLL(_LIB_PATH)
    lib.apxref_setup_last_error.restype = ctypes.c_char_p
    lib.apxref_factorize.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_uint, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]
    lib.apxref_factor_info.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
    lib.apxref_factor_copy.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
    lib.apxref_factor_free.argtypes = [ctypes.c_void_p]
    _lib = lib
    return lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def factorize(mat, seed: int = 0, threads: int = DEFAULT_THREADS, storage: int = 3) -> Factor:
    """Run the reference factorization on a gen.Matrix (full symmetric CSC)."""
    lib = _load()
    colptr = np.ascontiguousarray(mat.colptr, dtype=np.int32)
    rowidx = np.ascontiguousarray(mat.rowidx, dtype=np.int32)
    vals = np.ascontiguousarray(mat.vals, dtype=np.float64)
    h = ctypes.c_void_p()
    rc = lib.apxref_factorize(mat.n, _ptr(colptr), _ptr(rowidx), _ptr(vals), seed, threads, storage,
                              ctypes.byref(h))
    if rc != 0:
        raise RuntimeError("apxchol factorize failed: " + lib.apxref_setup_last_error().decode())
    try:
        n = ctypes.c_uint32(); nnz = ctypes.c_uint64(); sddm = ctypes.c_int()
        nr = ctypes.c_uint32(); lumped = ctypes.c_int64()
        lib.apxref_factor_info(h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(sddm),
                               ctypes.byref(nr), ctypes.byref(lumped))
        f = Factor(n=n.value, colptr=np.empty(n.value + 1, np.uint32),
                   rowidx=np.empty(nnz.value, np.uint32), vals=np.empty(nnz.value, np.float32),
                   perm=np.empty(n.value, np.uint32), sddm=bool(sddm.value),
                   rounds=np.empty(nr.value, np.uint64), lumped=lumped.value)
        lib.apxref_factor_copy(h, _ptr(f.colptr), _ptr(f.rowidx), _ptr(f.vals), _ptr(f.perm),
                               _ptr(f.rounds) if nr.value else None)
    finally:
        lib.apxref_factor_free(h)
    return f
