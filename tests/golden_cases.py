"""Loader of tests/golden/golden.npz (see tests/golden/make_golden.py)."""
import functools
import os

import numpy as np

from apxchol_b200.gen import Matrix
from apxchol_b200.refsetup import Factor

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
NAMES = ["grid2d_32", "grid3d_10", "regular_500", "rmat_9"]


@functools.lru_cache(maxsize=None)
def _data():
    return dict(np.load(PATH))


def case(name):
    d = _data()
    g = {k.split("/", 1)[1]: v for k, v in d.items() if k.startswith(name + "/")}
    n = int(g["n"])
    A = Matrix(n=n, colptr=g["a_colptr"], rowidx=g["a_rowidx"], vals=g["a_vals"], name=name)
    F = Factor(n=n, colptr=g["f_colptr"], rowidx=g["f_rowidx"], vals=g["f_vals"], perm=g["f_perm"],
               sddm=bool(g["f_sddm"]), rounds=g["f_rounds"])
    return A, F, g
