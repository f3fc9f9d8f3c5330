"""Seeded synthetic systems for the solve phase.

Every generator is deterministic for its seed (numpy PCG64 streams, drawn in
the order documented per function) and returns the operator as a full
symmetric CSC matrix (int32 column pointers / row indices, float64 values,
rows ascending in each column) -- the layout of the
`Eigen::SparseMatrix<double>` the reference's `apxchol::solve` takes
(include/apxchol/solver/solve.h:138-140).

A graph Laplacian L = D - W is singular (rank n-1); adding a positive
diagonal excess makes it SDDM (full rank), which the reference detects
itself (factorization_impl.h:704).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Matrix:
    """Full symmetric CSC operator."""
    n: int
    colptr: np.ndarray   # int32[n+1]
    rowidx: np.ndarray   # int32[nnz]
    vals: np.ndarray     # float64[nnz]
    name: str = ""
    sddm: bool = False   # True when a positive diagonal excess was added

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csc_matrix((self.vals, self.rowidx, self.colptr), shape=(self.n, self.n))

    def matvec(self, x: np.ndarray) -> np.ndarray:
        return self.to_scipy() @ x


def _laplacian(n: int, u: np.ndarray, v: np.ndarray, w: np.ndarray,
               excess: np.ndarray | None, name: str) -> Matrix:
    """L = D - W (+ diag(excess)) from an undirected edge list (u != v).
    Duplicate edges are merged with their weights summed."""
    import scipy.sparse as sp
    u = np.asarray(u, dtype=np.int64)
    v = np.asarray(v, dtype=np.int64)
    w = np.asarray(w, dtype=np.float64)
    if np.any(u == v):
        raise ValueError("self loops are not allowed")
    rows = np.concatenate([u, v])
    cols = np.concatenate([v, u])
    vals = np.concatenate([-w, -w])
    W = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsc()
    W.sum_duplicates()
    deg = -np.asarray(W.sum(axis=0)).ravel()
    diag = deg.copy()
    if excess is not None:
        diag = diag + excess
    L = (W + sp.diags(diag, 0, shape=(n, n), format="csc")).tocsc()
    L.sum_duplicates()
    L.sort_indices()
    return Matrix(n=n, colptr=L.indptr.astype(np.int32), rowidx=L.indices.astype(np.int32),
                  vals=L.data.astype(np.float64), name=name,
                  sddm=bool(excess is not None and np.any(excess > 0)))


def grid2d(nx: int, ny: int | None = None, seed: int = 0, wlo: float = 1.0, whi: float = 2.0,
           shift: float = 0.0) -> Matrix:
    """2D 5-point grid, vertex (i, j) = i + nx*j. Weights i.i.d. U[wlo, whi):
    first all x-edges in vertex order, then all y-edges. `shift` adds
    shift*degree to every diagonal entry (SDDM)."""
    ny = nx if ny is None else ny
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.arange(nx * ny).reshape(ny, nx)
    ux, vx = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    uy, vy = idx[:-1, :].ravel(), idx[1:, :].ravel()
    u = np.concatenate([ux, uy]); v = np.concatenate([vx, vy])
    w = rng.uniform(wlo, whi, size=u.size)
    excess = None
    if shift > 0:
        deg = np.bincount(np.concatenate([u, v]), minlength=nx * ny).astype(np.float64)
        excess = shift * deg
    return _laplacian(nx * ny, u, v, w, excess, f"grid2d_{nx}x{ny}")


def grid3d(n: int, seed: int = 1, log10_lo: float = -3.0, log10_hi: float = 3.0,
           boundary_excess: float = 1.0) -> Matrix:
    """3D 7-point grid n^3, vertex (i, j, k) = i + n*j + n^2*k. Weights
    10**U[log10_lo, log10_hi) (high contrast), drawn x-edges, then y, then z,
    each in vertex order. `boundary_excess` is added to the diagonal of every
    vertex on the cube's surface (SDDM)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.arange(n ** 3).reshape(n, n, n)          # [k, j, i]
    ux, vx = idx[:, :, :-1].ravel(), idx[:, :, 1:].ravel()
    uy, vy = idx[:, :-1, :].ravel(), idx[:, 1:, :].ravel()
    uz, vz = idx[:-1, :, :].ravel(), idx[1:, :, :].ravel()
    u = np.concatenate([ux, uy, uz]); v = np.concatenate([vx, vy, vz])
    w = 10.0 ** rng.uniform(log10_lo, log10_hi, size=u.size)
    excess = None
    if boundary_excess:
        k, j, i = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        on = (i == 0) | (i == n - 1) | (j == 0) | (j == n - 1) | (k == 0) | (k == n - 1)
        excess = np.where(on.ravel(), boundary_excess, 0.0)
    return _laplacian(n ** 3, u, v, w, excess, f"grid3d_{n}")


def _largest_component(n: int, u: np.ndarray, v: np.ndarray):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import connected_components
    A = sp.coo_matrix((np.ones(u.size), (u, v)), shape=(n, n))
    ncomp, lab = connected_components(A, directed=False)
    big = np.bincount(lab).argmax()
    keep = lab == big
    newid = -np.ones(n, dtype=np.int64)
    newid[keep] = np.arange(int(keep.sum()))
    m = keep[u] & keep[v]
    return int(keep.sum()), newid[u[m]], newid[v[m]], m


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 2) -> Matrix:
    """R-MAT power-law graph on 2^scale vertices with edge_factor*2^scale
    sampled edges (quadrant probabilities a, b, c, d = 1-a-b-c, one uniform
    draw per edge per level, levels from the top bit down). Self loops are
    dropped, duplicates merged with weight = multiplicity, and the result is
    restricted to its largest connected component: a singular Laplacian."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nv = 1 << scale
    ne = edge_factor * nv
    u = np.zeros(ne, dtype=np.int64)
    v = np.zeros(ne, dtype=np.int64)
    ab, abc = a + b, a + b + c
    chunk = 1 << 22
    for s in range(0, ne, chunk):
        e = min(ne, s + chunk)
        uu = np.zeros(e - s, dtype=np.int64)
        vv = np.zeros(e - s, dtype=np.int64)
        for lvl in range(scale):
            r = rng.random(e - s)
            bit = 1 << (scale - 1 - lvl)
            uu += np.where(r >= ab, bit, 0)                      # quadrants c, d: lower half
            vv += np.where(((r >= a) & (r < ab)) | (r >= abc), bit, 0)  # quadrants b, d: right half
        u[s:e] = uu
        v[s:e] = vv
    keep = u != v
    u, v = u[keep], v[keep]
    lo, hi = np.minimum(u, v), np.maximum(u, v)
    key = lo * nv + hi
    key, mult = np.unique(key, return_counts=True)
    lo, hi = key // nv, key % nv
    n, lo2, hi2, m = _largest_component(nv, lo, hi)
    return _laplacian(n, lo2, hi2, mult[m].astype(np.float64), None, f"rmat_{scale}_lcc")


def random_regular(n: int, degree: int = 6, seed: int = 0, wlo: float = 0.5, whi: float = 2.0,
                   shift: float = 0.0) -> Matrix:
    """Random `degree`-regular graph as the union of degree/2 random
    Hamiltonian cycles (one permutation each, drawn in order); an edge drawn
    twice is merged (weights summed), so a few vertices can have fewer than
    `degree` distinct neighbours. Weights U[wlo, whi) drawn after the cycles.
    `shift` adds shift*degree to the diagonal (SDDM)."""
    if degree % 2:
        raise ValueError("degree must be even")
    rng = np.random.Generator(np.random.PCG64(seed))
    us, vs = [], []
    for _ in range(degree // 2):
        p = rng.permutation(n)
        us.append(p); vs.append(np.roll(p, -1))
    u = np.concatenate(us); v = np.concatenate(vs)
    w = rng.uniform(wlo, whi, size=u.size)
    excess = None
    if shift > 0:
        deg = np.bincount(np.concatenate([u, v]), minlength=n).astype(np.float64)
        excess = shift * deg
    return _laplacian(n, u, v, w, excess, f"regular{degree}_{n}")


def rhs(n: int, seed: int, zero_mean: bool) -> np.ndarray:
    """N(0,1) right-hand side; projected to zero mean for a Laplacian."""
    rng = np.random.Generator(np.random.PCG64(seed))
    b = rng.standard_normal(n)
    if zero_mean:
        b = b - b.mean()
    return b
