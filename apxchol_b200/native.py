"""ctypes binding of the C ABI in include/apxb200.h (libapxb200.so).

The CUDA library is the only implementation of the solve phase in this
package: if it is missing, every entry point raises instead of falling back
to anything else.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libapxb200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "apxb200.h")

TRUE_RESIDUAL = 8
OK = 0
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_BAD_FACTOR, ERR_NONFINITE, ERR_BUDGET, ERR_BUSY = range(-1, -9, -1)
PREC_FP64, PREC_FP32, PREC_FP16 = 0, 1, 2
DEVICE_PTRS, CENTER_SCHEDULE, CENTER_ALWAYS, CENTER_NEVER = 1, 0, 2, 4

c_p = ctypes.c_void_p
_lib = None


class ApxbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"apxb error {code}: {msg}")
        self.code = code


class FactorInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("m", ctypes.c_uint32), ("nnz_factor", ctypes.c_uint64),
                ("nnz_stored", ctypes.c_uint64), ("dropped", ctypes.c_uint64),
                ("fwd_levels", ctypes.c_int32), ("bck_levels", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("sddm", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64), ("apply_count", ctypes.c_uint64),
                ("drop_rel", ctypes.c_double), ("dropped_flush", ctypes.c_uint64),
                ("sweep_grid", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class PcgResult(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("status", ctypes.c_int32), ("residual", ctypes.c_double),
                ("true_residual", ctypes.c_double), ("seconds", ctypes.c_double)]


# name -> (restype, argtypes)
_SIGS = {
    "apxb_last_error": (ctypes.c_char_p, []),
    "apxb_version": (ctypes.c_char_p, []),
    "apxb_engine_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(c_p)]),
    "apxb_engine_destroy": (ctypes.c_int, [c_p]),
    "apxb_engine_sync": (ctypes.c_int, [c_p]),
    "apxb_engine_stream": (c_p, [c_p]),
    "apxb_engine_set_spin_budget": (ctypes.c_int, [c_p, ctypes.c_uint64]),
    "apxb_engine_set_sweep_grid": (ctypes.c_int, [c_p, ctypes.c_int]),
    "apxb_engine_set_memory_budget": (ctypes.c_int, [c_p, ctypes.c_uint64]),
    "apxb_engine_memory_used": (ctypes.c_uint64, [c_p]),
    "apxb_factor_create": (ctypes.c_int, [c_p, ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.c_int, c_p,
                                          ctypes.c_uint32, ctypes.c_double, ctypes.c_int, ctypes.POINTER(c_p)]),
    "apxb_factor_destroy": (ctypes.c_int, [c_p]),
    "apxb_factor_info_get": (ctypes.c_int, [c_p, ctypes.POINTER(FactorInfo)]),
    "apxb_factor_arrays": (ctypes.c_int, [c_p] + [c_p] * 8),
    "apxb_factor_reset_apply_count": (ctypes.c_int, [c_p]),
    "apxb_prepare_host": (ctypes.c_int, [ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.c_int, c_p, ctypes.c_uint32,
                                         ctypes.c_double, c_p, c_p, c_p] + [c_p] * 8),
    "apxb_prepare_host_fp16": (ctypes.c_int, [ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.c_int, c_p, ctypes.c_uint32,
                                              ctypes.c_double, c_p, c_p] + [c_p] * 9),
    "apxb_sweep": (ctypes.c_int, [c_p, c_p, ctypes.c_int, c_p, c_p]),
    "apxb_sweep_pair": (ctypes.c_int, [c_p, c_p, c_p, c_p]),
    "apxb_sweep_pair_host": (ctypes.c_int, [c_p, c_p, c_p, c_p]),
    "apxb_sweep_pair_timed": (ctypes.c_int, [c_p, c_p, c_p, c_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "apxb_sweep_pair_multi": (ctypes.c_int, [c_p, c_p, ctypes.c_int, c_p, c_p]),
    "apxb_sweep_pair_noalloc": (ctypes.c_int, [c_p, c_p, c_p, c_p]),
    "apxb_apply": (ctypes.c_int, [c_p, c_p, c_p, c_p, ctypes.c_int, c_p]),
    "apxb_operator_create": (ctypes.c_int, [c_p, ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.POINTER(c_p)]),
    "apxb_operator_destroy": (ctypes.c_int, [c_p]),
    "apxb_operator_fp32": (ctypes.c_int, [c_p, ctypes.POINTER(ctypes.c_int)]),
    "apxb_operator_matvec": (ctypes.c_int, [c_p, c_p, c_p, c_p]),
    "apxb_pcg": (ctypes.c_int, [c_p, c_p, c_p, c_p, c_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.POINTER(PcgResult)]),
    "apxb_test_stalled_sweep": (ctypes.c_int, [c_p, c_p, ctypes.c_uint64]),
    "apxb_test_prep_compare": (ctypes.c_int, [c_p, ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.c_int, c_p,
                                              ctypes.c_uint32, ctypes.c_double, ctypes.c_int, c_p, c_p, c_p]),
    "apxb_batch_create": (ctypes.c_int, [c_p, ctypes.c_int, c_p, c_p, ctypes.c_int, ctypes.POINTER(c_p)]),
    "apxb_batch_plan_host": (ctypes.c_int, [ctypes.c_uint32, c_p, c_p, c_p, c_p, ctypes.c_int, c_p, ctypes.c_uint32,
                                            ctypes.c_double, ctypes.c_int, c_p, c_p]),
    "apxb_batch_destroy": (ctypes.c_int, [c_p]),
    "apxb_batch_size": (ctypes.c_int, [c_p, c_p, c_p, c_p]),
    "apxb_batch_solve": (ctypes.c_int, [c_p, c_p, c_p, c_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, c_p]),
    "apxb_batch_set_refresh": (ctypes.c_int, [c_p, ctypes.c_int]),
    "apxb_batch_admit": (ctypes.c_int, [c_p, ctypes.c_int, c_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "apxb_batch_step": (ctypes.c_int, [c_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]),
    "apxb_batch_query": (ctypes.c_int, [c_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]),
    "apxb_batch_slots": (ctypes.c_int, [c_p, ctypes.c_int64, c_p, c_p, c_p, c_p]),
    "apxb_batch_retire": (ctypes.c_int, [c_p, ctypes.c_int, c_p, ctypes.c_int]),
    "apxb_batch_retired": (ctypes.c_int, [c_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "apxb_batch_sweep_timed": (ctypes.c_int, [c_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_double)]),
}


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(apxb_[a-z_0-9]+)\s*\(", text, re.M)))


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library missing: {LIB_PATH} (build it with __graft_entry__.build())")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != OK:
        raise ApxbError(rc, load().apxb_last_error().decode())


def ptr(a):
    """Address of a numpy array (host) or a torch tensor (device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Engine:
    """apxb_engine: one GPU, one stream, an error word and workspaces."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = c_p()
        check(self.lib.apxb_engine_create(device, ctypes.byref(h)))
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.apxb_engine_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def sync(self):
        check(self.lib.apxb_engine_sync(self.h))

    @property
    def stream(self) -> int:
        return self.lib.apxb_engine_stream(self.h) or 0

    def set_spin_budget(self, ns: int):
        check(self.lib.apxb_engine_set_spin_budget(self.h, int(ns)))

    def set_sweep_grid(self, blocks: int):
        check(self.lib.apxb_engine_set_sweep_grid(self.h, int(blocks)))

    def set_memory_budget(self, nbytes: int):
        check(self.lib.apxb_engine_set_memory_budget(self.h, int(nbytes)))

    def memory_used(self) -> int:
        return int(self.lib.apxb_engine_memory_used(self.h))


class DeviceFactor:
    """apxb_factor: the reference factor prepared and resident on the GPU
    (the replacement of cuda_sptrsv::setup, sptrsv/cuda.h:233-459)."""

    def __init__(self, eng: Engine, fac, precision: int = PREC_FP64, drop_rel: float = -1.0):
        self.eng, self.lib = eng, eng.lib
        self._keep = [np.ascontiguousarray(fac.colptr, np.uint32), np.ascontiguousarray(fac.rowidx, np.uint32),
                      np.ascontiguousarray(fac.vals, np.float32), np.ascontiguousarray(fac.perm, np.uint32),
                      np.ascontiguousarray(fac.rounds, np.uint64)]
        cp_, ri, va, pe, ro = self._keep
        h = c_p()
        check(self.lib.apxb_factor_create(eng.h, fac.n, ptr(cp_), ptr(ri), ptr(va), ptr(pe), int(fac.sddm),
                                          ptr(ro) if ro.size else None, ro.size, drop_rel, precision,
                                          ctypes.byref(h)))
        self.h = h
        self._keep = None
        self.info = self.get_info()
        self.n, self.m, self.sddm = self.info.n, self.info.m, bool(self.info.sddm)

    def get_info(self) -> FactorInfo:
        inf = FactorInfo()
        check(self.lib.apxb_factor_info_get(self.h, ctypes.byref(inf)))
        return inf

    def close(self):
        if getattr(self, "h", None):
            self.lib.apxb_factor_destroy(self.h)
            self.h = None

    __del__ = close

    def arrays(self):
        inf = self.info
        m, nnz = inf.m, inf.nnz_stored
        out = dict(csr_ptr=np.empty(m + 1, np.uint32), csr_idx=np.empty(nnz, np.uint32),
                   csr_val=np.empty(nnz, np.float32), csc_ptr=np.empty(m + 1, np.uint32),
                   csc_idx=np.empty(nnz, np.uint32), csc_val=np.empty(nnz, np.float32),
                   fwd_thin=np.empty(m, np.uint8), bck_thin=np.empty(m, np.uint8))
        check(self.lib.apxb_factor_arrays(self.h, *[ptr(out[k]) for k in
                                                    ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx",
                                                     "csc_val", "fwd_thin", "bck_thin")]))
        return out

    def reset_apply_count(self):
        check(self.lib.apxb_factor_reset_apply_count(self.h))

    # -- sweeps on device tensors (torch float64, length m or m*k) --
    def sweep(self, direction: int, d_in, d_out):
        check(self.lib.apxb_sweep(self.eng.h, self.h, direction, ptr(d_in), ptr(d_out)))

    def sweep_pair(self, d_in, d_out):
        check(self.lib.apxb_sweep_pair(self.eng.h, self.h, ptr(d_in), ptr(d_out)))

    def sweep_pair_timed(self, d_in, d_out, reps: int) -> float:
        sec = ctypes.c_double()
        check(self.lib.apxb_sweep_pair_timed(self.eng.h, self.h, ptr(d_in), ptr(d_out), reps, ctypes.byref(sec)))
        return sec.value

    def sweep_pair_multi(self, k: int, d_in, d_out):
        check(self.lib.apxb_sweep_pair_multi(self.eng.h, self.h, k, ptr(d_in), ptr(d_out)))

    def sweep_pair_host(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        out = np.empty(self.m)
        check(self.lib.apxb_sweep_pair_host(self.eng.h, self.h, ptr(x), ptr(out)))
        return out

    def apply(self, b: np.ndarray, flags: int = CENTER_SCHEDULE):
        """z = M^-1 b in the original ordering (apx_cholesky::apply_core); returns (z, b.z)."""
        b = np.ascontiguousarray(b, np.float64)
        z = np.empty(self.n)
        rz = ctypes.c_double()
        check(self.lib.apxb_apply(self.eng.h, self.h, ptr(b), ptr(z), flags, ctypes.byref(rz)))
        return z, rz.value


class DeviceOperator:
    """apxb_operator: A in the factor's permuted ordering (cuda_pcg::setup, pcg_cuda.h:68-152)."""

    def __init__(self, eng: Engine, mat, perm):
        self.eng, self.lib = eng, eng.lib
        cp_ = np.ascontiguousarray(mat.colptr, np.int32)
        ri = np.ascontiguousarray(mat.rowidx, np.int32)
        va = np.ascontiguousarray(mat.vals, np.float64)
        pe = np.ascontiguousarray(perm, np.uint32)
        h = c_p()
        check(self.lib.apxb_operator_create(eng.h, mat.n, ptr(cp_), ptr(ri), ptr(va), ptr(pe), ctypes.byref(h)))
        self.h = h
        self.n = mat.n

    def close(self):
        if getattr(self, "h", None):
            self.lib.apxb_operator_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def fp32(self) -> bool:
        """Whether the values are stored in fp32 (all fp32-exact, or forced by
        APXCHOL_GPU_FP32_OPERATOR at creation)."""
        v = ctypes.c_int()
        check(self.lib.apxb_operator_fp32(self.h, ctypes.byref(v)))
        return bool(v.value)

    def matvec(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.n)
        check(self.lib.apxb_operator_matvec(self.eng.h, self.h, ptr(x), ptr(y)))
        return y


def pcg(eng: Engine, fac: DeviceFactor, op: DeviceOperator, b, x=None, tol: float = 1e-8, max_iter: int = 500,
        device_ptrs: bool = False, true_residual: bool = True):
    """GPU-resident PCG with the reference cpu_solver's semantics. Returns (x, PcgResult)."""
    res = PcgResult()
    if device_ptrs:
        check(eng.lib.apxb_pcg(eng.h, fac.h, op.h, ptr(b), ptr(x), tol, max_iter, DEVICE_PTRS, int(true_residual),
                               ctypes.byref(res)))
        return x, res
    b = np.ascontiguousarray(b, np.float64)
    x = np.empty(op.n) if x is None else x
    check(eng.lib.apxb_pcg(eng.h, fac.h, op.h, ptr(b), ptr(x), tol, max_iter, 0, int(true_residual),
                           ctypes.byref(res)))
    return x, res


def prepare_host(fac, drop_rel: float = -1.0):
    """Host-only preparation through the C ABI (no GPU needed)."""
    lib = load()
    cp_ = np.ascontiguousarray(fac.colptr, np.uint32)
    ri = np.ascontiguousarray(fac.rowidx, np.uint32)
    va = np.ascontiguousarray(fac.vals, np.float32)
    pe = np.ascontiguousarray(fac.perm, np.uint32)
    ro = np.ascontiguousarray(fac.rounds, np.uint64)
    m = ctypes.c_uint32(); nnz = ctypes.c_uint64(); lv = np.zeros(2, np.int32)
    args = (fac.n, ptr(cp_), ptr(ri), ptr(va), ptr(pe), int(fac.sddm), ptr(ro) if ro.size else None, ro.size,
            drop_rel, ctypes.byref(m), ctypes.byref(nnz), ptr(lv))
    check(lib.apxb_prepare_host(*args, *([None] * 8)))
    M, N = m.value, nnz.value
    out = dict(csr_ptr=np.empty(M + 1, np.uint32), csr_idx=np.empty(N, np.uint32), csr_val=np.empty(N, np.float32),
               csc_ptr=np.empty(M + 1, np.uint32), csc_idx=np.empty(N, np.uint32), csc_val=np.empty(N, np.float32),
               fwd_thin=np.empty(M, np.uint8), bck_thin=np.empty(M, np.uint8))
    check(lib.apxb_prepare_host(*args, *[ptr(out[k]) for k in ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx",
                                                                "csc_val", "fwd_thin", "bck_thin")]))
    out["m"], out["nnz"], out["levels"] = M, N, (int(lv[0]), int(lv[1]))
    return out


def prepare_host_fp16(fac, drop_rel: float = -1.0):
    """Host-only fp16 factor storage through the C ABI (no GPU): the arrays an
    APXB_PREC_FP16 factor uploads (binary16 values as uint16 bit patterns)."""
    lib = load()
    cp_ = np.ascontiguousarray(fac.colptr, np.uint32)
    ri = np.ascontiguousarray(fac.rowidx, np.uint32)
    va = np.ascontiguousarray(fac.vals, np.float32)
    pe = np.ascontiguousarray(fac.perm, np.uint32)
    ro = np.ascontiguousarray(fac.rounds, np.uint64)
    m = ctypes.c_uint32(); nnz = ctypes.c_uint64()
    args = (fac.n, ptr(cp_), ptr(ri), ptr(va), ptr(pe), int(fac.sddm), ptr(ro) if ro.size else None, ro.size,
            drop_rel, ctypes.byref(m), ctypes.byref(nnz))
    check(lib.apxb_prepare_host_fp16(*args, *([None] * 9)))
    M, N = m.value, nnz.value
    out = dict(csc_ptr=np.empty(M + 1, np.uint32), csc_idx=np.empty(N, np.uint32), csc_val16=np.empty(N, np.uint16),
               csr_ptr=np.empty(M + 1, np.uint32), csr_idx=np.empty(N, np.uint32), csr_val16=np.empty(N, np.uint16),
               diag=np.empty(M, np.float32), inv_scale=np.empty(M, np.float32), stats=np.zeros(3, np.uint64))
    check(lib.apxb_prepare_host_fp16(*args, *[ptr(out[k]) for k in ("csc_ptr", "csc_idx", "csc_val16", "csr_ptr",
                                                                     "csr_idx", "csr_val16", "diag", "inv_scale",
                                                                     "stats")]))
    out["m"], out["nnz"] = M, N
    return out


def batch_plan_host(fac, k: int, drop_rel: float = -1.0):
    """Host-only build + check of the batch sweep plans (no GPU): ((items fwd, bck), (chunks fwd, bck))."""
    lib = load()
    cp_ = np.ascontiguousarray(fac.colptr, np.uint32)
    ri = np.ascontiguousarray(fac.rowidx, np.uint32)
    va = np.ascontiguousarray(fac.vals, np.float32)
    pe = np.ascontiguousarray(fac.perm, np.uint32)
    ro = np.ascontiguousarray(fac.rounds, np.uint64)
    items, chunks = np.zeros(2, np.uint32), np.zeros(2, np.uint32)
    check(lib.apxb_batch_plan_host(fac.n, ptr(cp_), ptr(ri), ptr(va), ptr(pe), int(fac.sddm),
                                   ptr(ro) if ro.size else None, ro.size, drop_rel, k, ptr(items), ptr(chunks)))
    return tuple(int(v) for v in items), tuple(int(v) for v in chunks)


class Batch:
    """apxb_batch: S instances x k right-hand-side slots solved together
    (fp32 preconditioner sweeps, fp64 everything else)."""

    def __init__(self, eng: Engine, factors, operators, k: int):
        self.eng, self.lib = eng, eng.lib
        self.factors, self.operators = list(factors), list(operators)   # keep alive
        S = len(self.factors)
        fa = (c_p * S)(*[f.h for f in self.factors])
        oa = (c_p * S)(*[o.h for o in self.operators])
        h = c_p()
        check(self.lib.apxb_batch_create(eng.h, S, fa, oa, k, ctypes.byref(h)))
        self.h = h
        self.S, self.k = S, k
        self.sizes = [f.n for f in self.factors]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n_total = int(self.offsets[-1])

    def close(self):
        if getattr(self, "h", None):
            self.lib.apxb_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def pack(self, rhs):
        """rhs[i] = array (n_i,) or (c_i, n_i) -> flat caller layout and nrhs."""
        B = np.zeros(self.n_total * self.k)
        nrhs = np.zeros(self.S, np.int32)
        for i, bi in enumerate(rhs):
            bi = np.atleast_2d(np.asarray(bi, np.float64))
            c, ni = bi.shape
            assert ni == self.sizes[i] and c <= self.k
            base = self.k * int(self.offsets[i])
            B[base: base + c * ni] = bi.ravel()
            nrhs[i] = c
        return B, nrhs

    def unpack(self, X, nrhs):
        out = []
        for i in range(self.S):
            base, ni = self.k * int(self.offsets[i]), self.sizes[i]
            out.append(X[base: base + int(nrhs[i]) * ni].reshape(int(nrhs[i]), ni))
        return out

    def solve(self, rhs, tol=1e-8, max_iter=500, true_residual=True):
        """rhs: list per instance of (c_i, n_i) arrays. Returns (list of x
        arrays, list of per-instance result lists)."""
        B, nrhs = self.pack(rhs)
        X = np.empty_like(B)
        res = (PcgResult * (self.S * self.k))()
        flags = TRUE_RESIDUAL if true_residual else 0
        check(self.lib.apxb_batch_solve(self.h, ptr(B), ptr(X), ptr(nrhs), tol, max_iter, flags, res))
        results = [[res[i * self.k + c] for c in range(int(nrhs[i]))] for i in range(self.S)]
        return self.unpack(X, nrhs), results

    def solve_raw(self, B, X, nrhs, tol=1e-8, max_iter=500, flags=0):
        """Caller-layout buffers (numpy host or torch device with DEVICE_PTRS)."""
        res = (PcgResult * (self.S * self.k))()
        check(self.lib.apxb_batch_solve(self.h, ptr(B), ptr(X), ptr(nrhs), tol, max_iter, flags, res))
        return res

    def set_refresh(self, every: int):
        """Recompute a slot's residual as b - A x (fp64) every `every` of its iterations, and once more to
        confirm convergence before a slot stops (0: never; the recurrence alone then stops a slot)."""
        check(self.lib.apxb_batch_set_refresh(self.h, every))

    # -- continuous batching (every call enqueues and returns) --
    def admit(self, slot: int, b, tol: float = 1e-8, max_iter: int = 500, device_ptrs: bool = False):
        """Load a right-hand side (the slot's instance size, original ordering)
        into an idle slot. Pinned host or device memory is read later in stream
        order: keep it unchanged until the next step has finished."""
        if not device_ptrs and isinstance(b, np.ndarray):
            b = np.ascontiguousarray(b, np.float64)
            assert b.shape == (self.sizes[slot // self.k],)
        check(self.lib.apxb_batch_admit(self.h, slot, ptr(b), tol, max_iter, DEVICE_PTRS if device_ptrs else 0))

    def step(self, iterations: int = 1) -> int:
        """Enqueue PCG iterations of every live slot; returns the step id."""
        sid = ctypes.c_int64()
        check(self.lib.apxb_batch_step(self.h, iterations, ctypes.byref(sid)))
        return sid.value

    def ready(self, step_id: int) -> bool:
        r = ctypes.c_int()
        check(self.lib.apxb_batch_query(self.h, step_id, ctypes.byref(r)))
        return bool(r.value)

    def slots(self, step_id: int):
        """(done, iterations, status, residual) arrays after step step_id."""
        ns = self.S * self.k
        done, its, st = (np.zeros(ns, np.int32) for _ in range(3))
        res = np.zeros(ns)
        check(self.lib.apxb_batch_slots(self.h, step_id, ptr(done), ptr(its), ptr(st), ptr(res)))
        return done.astype(bool), its, st, res

    def retire(self, slot: int, x=None, device_ptrs: bool = False):
        """Enqueue the copy of a finished slot's solution into x (returned);
        read it once retired(slot) is true."""
        if x is None:
            x = np.empty(self.sizes[slot // self.k])
        check(self.lib.apxb_batch_retire(self.h, slot, ptr(x), DEVICE_PTRS if device_ptrs else 0))
        return x

    def retired(self, slot: int) -> bool:
        r = ctypes.c_int()
        check(self.lib.apxb_batch_retired(self.h, slot, ctypes.byref(r)))
        return bool(r.value)

    def sweep_timed(self, reps: int = 10):
        """Seconds per forward and per backward fp32 sweep of this batch (CUDA events)."""
        f, b = ctypes.c_double(), ctypes.c_double()
        check(self.lib.apxb_batch_sweep_timed(self.h, reps, ctypes.byref(f), ctypes.byref(b)))
        return f.value, b.value
