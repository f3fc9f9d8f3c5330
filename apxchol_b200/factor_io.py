"""Factor files: save a factorization once, load it later and solve from numpy.

A factor file is a numpy .npz archive holding the fields of
apxchol::factorization that the solve phase consumes
(include/apxchol/solver/factorization.h:22-56): the lower-triangular CSC
factor (u32 column pointers and row indices, f32 values, diagonal first in
each column, rows ascending), the elimination permutation
perm[original] = position, the SDDM flag and the per-round independent-set
sizes, plus a format version. Loading checks the shapes and dtypes; the
factor's structure is checked again by apxb_factor_create.
"""
from __future__ import annotations

import numpy as np

from .refsetup import Factor

FORMAT = "apxb200-factor-v1"


def save_factor(path, fac: Factor) -> None:
    np.savez(path, format=np.array(FORMAT), n=np.array(fac.n, np.uint64),
             colptr=np.ascontiguousarray(fac.colptr, np.uint32), rowidx=np.ascontiguousarray(fac.rowidx, np.uint32),
             vals=np.ascontiguousarray(fac.vals, np.float32), perm=np.ascontiguousarray(fac.perm, np.uint32),
             sddm=np.array(bool(fac.sddm)), rounds=np.ascontiguousarray(fac.rounds, np.uint64),
             lumped=np.array(int(fac.lumped), np.int64))


def load_factor(path) -> Factor:
    with np.load(path, allow_pickle=False) as z:
        if str(z["format"]) != FORMAT:
            raise ValueError(f"{path}: not a {FORMAT} file")
        n = int(z["n"])
        colptr, rowidx, vals, perm = z["colptr"], z["rowidx"], z["vals"], z["perm"]
        if colptr.dtype != np.uint32 or rowidx.dtype != np.uint32 or vals.dtype != np.float32 or perm.dtype != np.uint32:
            raise ValueError(f"{path}: unexpected array types")
        if colptr.shape != (n + 1,) or perm.shape != (n,) or rowidx.shape != vals.shape or \
                rowidx.shape != (int(colptr[-1]),):
            raise ValueError(f"{path}: inconsistent array sizes")
        return Factor(n=n, colptr=colptr, rowidx=rowidx, vals=vals, perm=perm, sddm=bool(z["sddm"]),
                      rounds=z["rounds"].astype(np.uint64), lumped=int(z["lumped"]))
