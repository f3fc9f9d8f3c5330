"""Generates tests/golden/golden.npz: outputs of the apxchol reference itself
(its factorization, omp_sptrsv sweeps, apx_cholesky apply and cpu_solver PCG,
compiled from the reference sources into oracle/_ref and
apxchol_b200/refsetup/_ref) on small seeded systems, with one OpenMP thread.

Run from the repository root where the reference builds exist:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from apxchol_b200 import gen, refsetup  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "grid2d_32": (lambda: gen.grid2d(32, seed=0), 0),
    "grid3d_10": (lambda: gen.grid3d(10, seed=1), 0),
    "regular_500": (lambda: gen.random_regular(500, seed=3, shift=1e-3), 1),
    "rmat_9": (lambda: gen.rmat(9, seed=2), 2),
}


def main():
    out = {}
    oracle.set_threads(1)
    for name, (build, seed) in CASES.items():
        A = build()
        F = refsetup.factorize(A, seed=seed, threads=1)
        R = oracle.Ref(A, F)
        rng = np.random.default_rng(7)
        x = rng.standard_normal(F.m)
        b = gen.rhs(A.n, 11, not F.sddm)
        y = R.forward(x)
        z = R.transpose(y)
        za = R.apply(b)                           # Eigen-seam application, counter reset first
        zf, rz = R.apply_fused(b, float(b.sum())) # PCG-entry application
        xs, it, res, _ = R.solve(b, 1e-8, 500)
        arr = R.arrays()
        p = f"{name}/"
        out.update({
            p + "a_colptr": A.colptr, p + "a_rowidx": A.rowidx, p + "a_vals": A.vals,
            p + "f_colptr": F.colptr, p + "f_rowidx": F.rowidx, p + "f_vals": F.vals, p + "f_perm": F.perm,
            p + "f_rounds": F.rounds, p + "f_sddm": np.array(F.sddm), p + "n": np.array(A.n),
            p + "x": x, p + "fwd": y, p + "pair": z, p + "b": b, p + "apply": za, p + "apply_fused": zf,
            p + "rz": np.array(rz), p + "pcg_x": xs, p + "pcg_iters": np.array(it), p + "pcg_res": np.array(res),
            p + "csr_ptr": arr["csr_ptr"], p + "csr_idx": arr["csr_idx"], p + "csr_val": arr["csr_val"],
            p + "csc_ptr": arr["csc_ptr"], p + "csc_idx": arr["csc_idx"], p + "csc_val": arr["csc_val"],
        })
        print(f"{name}: n={A.n} nnz(L)={F.nnz} stored={R.nnz_stored} pcg iters={it} res={res:.3e}")
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz"), **out)


if __name__ == "__main__":
    main()
