"""Seeded test systems shared by the tests (built once per process)."""
import functools

from apxchol_b200 import gen, refsetup

# name -> (builder, factor seed)
SPECS = {
    "grid2d_64": (lambda: gen.grid2d(64, seed=0), 0),                       # Laplacian
    "grid2d_256": (lambda: gen.grid2d(256, seed=0), 0),                     # Laplacian (small C1 shape)
    "grid3d_24": (lambda: gen.grid3d(24, seed=1), 0),                       # SDDM, high contrast
    "grid3d_48": (lambda: gen.grid3d(48, seed=1), 1),                       # SDDM, high contrast
    "regular_3000": (lambda: gen.random_regular(3000, seed=3, shift=1e-3), 1),  # SDDM
    "rmat_12": (lambda: gen.rmat(12, seed=2), 2),                           # Laplacian, power law
    "rmat_14": (lambda: gen.rmat(14, seed=2), 2),                           # Laplacian, one 3676-entry row
    "path_200": (lambda: gen.grid2d(200, 1, seed=5), 0),                    # Laplacian, a path
}


@functools.lru_cache(maxsize=None)
def problem(name: str, threads: int = refsetup.DEFAULT_THREADS):
    build, seed = SPECS[name]
    A = build()
    F = refsetup.factorize(A, seed=seed, threads=threads)
    return A, F
