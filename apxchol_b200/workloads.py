"""The synthetic benchmark workloads, built with this project's seeded
generators (apxchol_b200.gen) and the reference's factorization.

  grid3d_128      3D 7-point 128^3, weights 10^U[-3,3] (seed 1), +1 on the
                  boundary diagonal (SDDM); factor seed 1.
  rmat_22         R-MAT scale 22, 16 * 2^22 sampled edges, (a,b,c,d) =
                  (.57,.19,.19,.05), seed 2; self loops dropped, duplicates
                  merged with weight = multiplicity, largest connected
                  component; singular Laplacian. Factor seed 2.
  instances_256   256 SDDM systems, n ~ U[1000, 200000]: even instances 2D
                  5-point grids (weights U[1,2]), odd ones random 6-regular
                  graphs (weights U[0.5,2]); diagonal shift 1e-3 * degree;
                  1-8 right-hand sides each (uniform).
  serving_8       8 matrices: 2 x 2D grid 1024^2, 2 x 3D grid 96^3,
                  2 x R-MAT scale 20 LCC, 2 x random 6-regular n = 500k;
                  weights as above, generator and factor seeds 10-17.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import gen, refsetup

FACTOR_THREADS = 8


def _factor(A, seed, log=None, name=""):
    t0 = time.time()
    F = refsetup.factorize(A, seed=seed, threads=FACTOR_THREADS)
    if log:
        log(f"[workload] {name}: n={A.n} nnz(A)={A.nnz} factor nnz={F.nnz} ({time.time() - t0:.1f}s)")
    return F


def grid3d_128(log=None):
    A = gen.grid3d(128, seed=1)
    return A, _factor(A, 1, log, "grid3d_128")


def rmat_22(log=None):
    A = gen.rmat(22, seed=2)
    return A, _factor(A, 2, log, "rmat_22")


def instances_256(log=None, count: int = 256, seed: int = 4):
    """[(A, F, n_rhs)] of the uneven multi-instance workload."""
    rng = np.random.default_rng(seed)
    out = []
    t0 = time.time()
    for i in range(count):
        n = int(rng.integers(1000, 200001))
        if i % 2 == 0:
            nx = max(2, int(round(math.sqrt(n))))
            A = gen.grid2d(nx, max(2, n // nx), seed=1000 + i, shift=1e-3)
        else:
            A = gen.random_regular(n, seed=1000 + i, shift=1e-3)
        F = refsetup.factorize(A, seed=1000 + i, threads=FACTOR_THREADS)
        out.append((A, F, int(rng.integers(1, 9))))
    if log:
        log(f"[workload] instances_256: sum n = {sum(a.n for a, _, _ in out)}, "
            f"right-hand sides = {sum(c for _, _, c in out)} ({time.time() - t0:.1f}s)")
    return out


def serving_8(log=None):
    """[(name, A, F)] of the serving workload."""
    specs = [("grid2d_1024_a", lambda: gen.grid2d(1024, seed=10), 10),
             ("grid2d_1024_b", lambda: gen.grid2d(1024, seed=11), 11),
             ("grid3d_96_a", lambda: gen.grid3d(96, seed=12), 12),
             ("grid3d_96_b", lambda: gen.grid3d(96, seed=13), 13),
             ("rmat_20_a", lambda: gen.rmat(20, seed=14), 14),
             ("rmat_20_b", lambda: gen.rmat(20, seed=15), 15),
             ("regular_500k_a", lambda: gen.random_regular(500_000, seed=16, shift=1e-3), 16),
             ("regular_500k_b", lambda: gen.random_regular(500_000, seed=17, shift=1e-3), 17)]
    out = []
    for name, build, seed in specs:
        A = build()
        out.append((name, A, _factor(A, seed, log, name)))
    return out
