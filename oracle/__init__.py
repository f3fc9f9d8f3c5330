"""TEST INFRASTRUCTURE: the CPU checkers of the solve phase.

Two libraries, both built by oracle/Makefile:
  * `Ref`  -- the apxchol reference's own CPU solve phase (cpu_solver +
    omp_sptrsv, src/solve.cpp and include/apxchol/solver/sptrsv/omp.h),
    compiled unchanged from its sources into _ref/libapxref.so;
  * `Oracle` -- the plain-C restatement in apxoracle.c, pinned byte-for-byte
    against `Ref` by tests/test_oracle_pin.py.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this package; the CUDA product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(_HERE, "_ref", "libapxref.so")
REF_LIB_V4 = os.path.join(_HERE, "_ref", "libapxref_v4.so")   # the same sources for x86-64-v4 (AVX-512)
ORACLE_LIB = os.path.join(_HERE, "_build", "liboracle.so")

c_p = ctypes.c_void_p


def _ptr(a):
    return None if a is None else a.ctypes.data


def build(ref_root: str | None = None) -> None:
    """Compile the checkers; the reference library only where the reference
    source tree (ref_root, else $APXCHOL_REF) is present."""
    import subprocess
    ref_root = ref_root or os.environ.get("APXCHOL_REF", "")
    targets = ["oracle"] + (["ref"] if ref_root and os.path.isdir(ref_root) else [])
    subprocess.check_call(["make", "-s", "-C", _HERE, f"REF={ref_root}"] + targets)


# --------------------------------------------------------------------- reference

_ref = None
_ref_path = REF_LIB

_V4_FLAGS = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def host_has_avx512() -> bool:
    """Whether this host runs x86-64-v4 code (the AVX-512 subsets it needs)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split(":", 1)[1].split())
                    return all(x in fl for x in _V4_FLAGS)
    except OSError:
        pass
    return False


def use_fastest_ref() -> str:
    """Load the x86-64-v4 build of the reference where this host supports it
    (the timed CPU baseline); else the portable build. Call before the first
    use of `Ref`. Returns the library's file name."""
    global _ref_path
    if _ref is None and os.path.exists(REF_LIB_V4) and host_has_avx512():
        _ref_path = REF_LIB_V4
    return os.path.basename(_ref_path)


def host_cores() -> int:
    """Physical cores this process may run on: the CPUs of its affinity mask
    divided by the hardware threads per core (the count OMP_NUM_THREADS is set
    to for the CPU baseline)."""
    avail = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        import psutil
        logical, physical = psutil.cpu_count(logical=True), psutil.cpu_count(logical=False)
        per_core = max(1, (logical or 1) // max(1, physical or 1))
    except Exception:
        per_core = 1
    return max(1, avail // per_core)


_ref_libs = {}


def _load_ref(path: str | None = None):
    """The reference library at `path` (default: the selected build), loaded once."""
    global _ref
    path = path or _ref_path
    if path not in _ref_libs:
        if not os.path.exists(path):
            raise RuntimeError(f"reference CPU library missing: {path}")
        lib = ctypes.CDLL(path)
        lib.apxref_last_error.restype = ctypes.c_char_p
        lib.apxref_set_threads.argtypes = [ctypes.c_int]
        lib.apxref_solver_create.argtypes = [ctypes.c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_p,
                                             ctypes.c_int, c_p, ctypes.c_uint32, ctypes.c_int,
                                             ctypes.POINTER(c_p)]
        lib.apxref_solver_free.argtypes = [c_p]
        lib.apxref_solve.argtypes = [c_p, c_p, c_p, ctypes.c_double, ctypes.c_int, c_p, c_p, c_p]
        lib.apxref_apply.argtypes = [c_p, c_p, c_p, ctypes.c_int]
        lib.apxref_apply_fused.argtypes = [c_p, c_p, ctypes.c_double, c_p, ctypes.c_int]
        lib.apxref_apply_fused.restype = ctypes.c_double
        lib.apxref_forward.argtypes = [c_p, c_p, c_p]
        lib.apxref_transpose.argtypes = [c_p, c_p, c_p]
        lib.apxref_pair_seconds.argtypes = [c_p, c_p, c_p, c_p, ctypes.c_int]
        lib.apxref_pair_seconds.restype = ctypes.c_double
        lib.apxref_sptrsv_info.argtypes = [c_p, c_p, c_p, c_p, c_p]
        lib.apxref_sptrsv_arrays.argtypes = [c_p] * 7
        lib.apxref_level_sizes.argtypes = [c_p, ctypes.c_int, c_p]
        lib.apxref_fp16_prep.argtypes = [ctypes.c_uint32, c_p, c_p, c_p, ctypes.c_int, ctypes.c_double,
                                         c_p, c_p] + [c_p] * 9
        _ref_libs[path] = lib
    if path == _ref_path:
        _ref = _ref_libs[path]
    return _ref_libs[path]


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def set_threads(t: int, lib_path: str | None = None) -> int:
    return _load_ref(lib_path).apxref_set_threads(t)


def fp16_prep(fac, rel=-1.0):
    """The reference GPU backend's fp16 factor storage, from its own host code
    (cuda_host.h:120-258 with the scale fallback of cuda.h:295-301): CSR(L^T)
    = CSC(L11) and CSR(L11) with binary16 values, diag, inv_scale and the drop
    and flush counts. rel < 0 means the default 1e-4."""
    lib = _load_ref()
    rel = DROP_REL if rel < 0 else rel
    cp_ = np.ascontiguousarray(fac.colptr, np.uint32)
    ri = np.ascontiguousarray(fac.rowidx, np.uint32)
    va = np.ascontiguousarray(fac.vals, np.float32)
    m = ctypes.c_uint32(); nnz = ctypes.c_uint64()
    args = (fac.n, _ptr(cp_), _ptr(ri), _ptr(va), int(fac.sddm), rel, ctypes.byref(m), ctypes.byref(nnz))
    if lib.apxref_fp16_prep(*args, *([None] * 9)):
        raise RuntimeError(lib.apxref_last_error().decode())
    M, N = m.value, nnz.value
    out = dict(csc_ptr=np.empty(M + 1, np.int32), csc_idx=np.empty(N, np.int32), csc_val16=np.empty(N, np.uint16),
               csr_ptr=np.empty(M + 1, np.int32), csr_idx=np.empty(N, np.int32), csr_val16=np.empty(N, np.uint16),
               diag=np.empty(M, np.float32), inv_scale=np.empty(M, np.float32), stats=np.zeros(3, np.uint64))
    if lib.apxref_fp16_prep(*args, *[_ptr(out[k]) for k in ("csc_ptr", "csc_idx", "csc_val16", "csr_ptr", "csr_idx",
                                                            "csr_val16", "diag", "inv_scale", "stats")]):
        raise RuntimeError(lib.apxref_last_error().decode())
    out["m"], out["nnz"] = M, N
    return out


class Ref:
    """The reference cpu_solver built on a given factor (cpu_solver(L, F),
    src/solve.cpp:295-318)."""

    def __init__(self, mat, fac, lib_path: str | None = None):
        lib = _load_ref(lib_path)
        self.lib = lib
        self.n = mat.n
        self._keep = [np.ascontiguousarray(a) for a in
                      (mat.colptr, mat.rowidx, mat.vals, fac.colptr, fac.rowidx, fac.vals, fac.perm,
                       fac.rounds)]
        a_p, a_i, a_v, f_p, f_i, f_v, perm, rounds = self._keep
        h = c_p()
        rc = lib.apxref_solver_create(mat.n, _ptr(a_p), _ptr(a_i), _ptr(a_v), _ptr(f_p), _ptr(f_i),
                                      _ptr(f_v), _ptr(perm), int(fac.sddm),
                                      _ptr(rounds) if rounds.size else None, rounds.size, 0,
                                      ctypes.byref(h))
        if rc != 0:
            raise RuntimeError("reference cpu_solver failed: " + lib.apxref_last_error().decode())
        self.h = h
        m = ctypes.c_uint32(); nnz = ctypes.c_uint64(); fl = ctypes.c_int(); bl = ctypes.c_int()
        lib.apxref_sptrsv_info(h, ctypes.byref(m), ctypes.byref(nnz), ctypes.byref(fl), ctypes.byref(bl))
        self.m, self.nnz_stored, self.fwd_levels, self.bck_levels = m.value, nnz.value, fl.value, bl.value

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.apxref_solver_free(self.h)
            self.h = None

    def solve(self, b, tol=1e-8, max_iter=500):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.n)
        it = ctypes.c_int(); res = ctypes.c_double(); secs = ctypes.c_double()
        rc = self.lib.apxref_solve(self.h, _ptr(b), _ptr(x), tol, max_iter, ctypes.byref(it),
                                   ctypes.byref(res), ctypes.byref(secs))
        if rc != 0:
            raise RuntimeError(self.lib.apxref_last_error().decode())
        return x, it.value, res.value, secs.value

    def apply(self, r, reset=True):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.n)
        self.lib.apxref_apply(self.h, _ptr(r), _ptr(z), int(reset))
        return z

    def apply_fused(self, r, r_sum, reset=True):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.n)
        rz = self.lib.apxref_apply_fused(self.h, _ptr(r), float(r_sum), _ptr(z), int(reset))
        return z, rz

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.m)
        self.lib.apxref_forward(self.h, _ptr(x), _ptr(y))
        return y

    def transpose(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        z = np.empty(self.m)
        self.lib.apxref_transpose(self.h, _ptr(y), _ptr(z))
        return z

    def pair_seconds(self, x, reps=5):
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.empty(self.m); z = np.empty(self.m)
        return self.lib.apxref_pair_seconds(self.h, _ptr(x), _ptr(t), _ptr(z), reps)

    def arrays(self):
        m, nnz = self.m, self.nnz_stored
        out = dict(csr_ptr=np.empty(m + 1, np.uint32), csr_idx=np.empty(nnz, np.uint32),
                   csr_val=np.empty(nnz, np.float32), csc_ptr=np.empty(m + 1, np.uint32),
                   csc_idx=np.empty(nnz, np.uint32), csc_val=np.empty(nnz, np.float32))
        self.lib.apxref_sptrsv_arrays(self.h, *[_ptr(out[k]) for k in
                                                ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx", "csc_val")])
        return out

    def level_sizes(self, fwd=True):
        s = np.empty(self.fwd_levels if fwd else self.bck_levels, np.int32)
        self.lib.apxref_level_sizes(self.h, int(fwd), _ptr(s))
        return s


# --------------------------------------------------------------------- restatement

_ora = None


class _System(ctypes.Structure):
    _fields_ = [("n", ctypes.c_uint32), ("a_ptr", c_p), ("a_idx", c_p), ("a_val", c_p),
                ("m", ctypes.c_uint32), ("sddm", ctypes.c_int32), ("perm", c_p),
                ("csr_ptr", c_p), ("csr_idx", c_p), ("csr_val", c_p),
                ("csc_ptr", c_p), ("csc_idx", c_p), ("csc_val", c_p),
                ("fwd_thin", c_p), ("bck_thin", c_p),
                ("nt", ctypes.c_int32), ("center_k", ctypes.c_int32), ("apply_count", ctypes.c_uint64)]


def _load_oracle():
    global _ora
    if _ora is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"oracle library missing: {ORACLE_LIB}")
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.ora_prepare.restype = ctypes.c_int64
        lib.ora_prepare.argtypes = [ctypes.c_uint32, ctypes.c_uint32, c_p, c_p, c_p, ctypes.c_double] + [c_p] * 6
        lib.ora_levels.restype = ctypes.c_int32
        lib.ora_levels.argtypes = [ctypes.c_uint32, c_p, c_p, c_p, c_p, c_p, ctypes.c_uint32, c_p, c_p, c_p]
        lib.ora_thin_flags.argtypes = [ctypes.c_uint32, c_p, ctypes.c_int32, ctypes.c_uint32, c_p]
        lib.ora_sweep.argtypes = [ctypes.c_int, ctypes.c_uint32, c_p, c_p, c_p, c_p, c_p, c_p]
        lib.ora_apply_core.restype = ctypes.c_double
        lib.ora_apply_core.argtypes = [ctypes.POINTER(_System), c_p, ctypes.c_double, ctypes.c_int, c_p, ctypes.c_int]
        lib.ora_apply_fused.restype = ctypes.c_double
        lib.ora_apply_fused.argtypes = [ctypes.POINTER(_System), c_p, ctypes.c_double, c_p]
        lib.ora_apply.argtypes = [ctypes.POINTER(_System), c_p, c_p]
        lib.ora_pcg.argtypes = [ctypes.POINTER(_System), c_p, ctypes.c_double, ctypes.c_int, c_p, c_p, c_p]
        lib.ora_sweep16.argtypes = [ctypes.c_int, ctypes.c_uint32] + [c_p] * 7
        _ora = lib
    return _ora


def sweep16(direction, h, rhs, in_scale=None):
    """One fp64 sweep over the fp16 storage h (apxchol_b200.native.prepare_host_fp16's
    arrays): the reference test's host sweep (test_sptrsv_drop.cpp:1100-1127).
    direction 0: forward over CSR(L11); 1: backward over CSC(L11), the right-hand
    side times in_scale (fp64) when given."""
    lib = _load_oracle()
    m = int(h["m"])
    key = "csr" if direction == 0 else "csc"
    ptr = np.ascontiguousarray(h[key + "_ptr"], np.uint32)
    idx = np.ascontiguousarray(h[key + "_idx"], np.uint32)
    v16 = np.ascontiguousarray(h[key + "_val16"], np.uint16)
    diag = np.ascontiguousarray(h["diag"], np.float32)
    r = np.ascontiguousarray(rhs, np.float64)
    sc = None if in_scale is None else np.ascontiguousarray(in_scale, np.float64)
    out = np.empty(m)
    lib.ora_sweep16(int(direction), m, _ptr(ptr), _ptr(idx), _ptr(v16), _ptr(diag),
                    _ptr(sc) if sc is not None else None, _ptr(r), _ptr(out))
    return out


THIN_THRESHOLD = 1024   # kSpTRSVOMPThreshold, include/apxchol/solver/sptrsv/omp.h:32
DROP_REL = 1e-4         # kFactorDropRelDefault, include/apxchol/solver/sptrsv/factor_drop.h:70


def prepare(fac, rel=DROP_REL):
    """Host prep + levels + per-row sum modes, as the reference's omp_sptrsv."""
    lib = _load_oracle()
    n, m = fac.n, fac.m
    cap = max(fac.nnz, 1)
    a = dict(csr_ptr=np.empty(m + 1, np.uint32), csr_idx=np.empty(cap, np.uint32),
             csr_val=np.empty(cap, np.float32), csc_ptr=np.empty(m + 1, np.uint32),
             csc_idx=np.empty(cap, np.uint32), csc_val=np.empty(cap, np.float32))
    nnz = lib.ora_prepare(n, m, _ptr(fac.colptr), _ptr(fac.rowidx), _ptr(fac.vals), rel,
                          *[_ptr(a[k]) for k in ("csr_ptr", "csr_idx", "csr_val", "csc_ptr", "csc_idx", "csc_val")])
    if nnz < 0:
        raise ValueError("malformed factor")
    for k in ("csr_idx", "csr_val", "csc_idx", "csc_val"):
        a[k] = a[k][:nnz].copy()
    fl = np.zeros(m, np.int32); bl = np.zeros(m, np.int32); nb = ctypes.c_int32()
    rounds = np.ascontiguousarray(fac.rounds, dtype=np.uint64)
    nf = lib.ora_levels(m, _ptr(a["csr_ptr"]), _ptr(a["csr_idx"]), _ptr(a["csc_ptr"]), _ptr(a["csc_idx"]),
                        _ptr(rounds) if rounds.size else None, rounds.size, _ptr(fl), _ptr(bl), ctypes.byref(nb))
    a["fwd_level"], a["bck_level"], a["n_fwd_levels"], a["n_bck_levels"] = fl, bl, nf, nb.value
    a["fwd_thin"] = np.empty(m, np.uint8); a["bck_thin"] = np.empty(m, np.uint8)
    lib.ora_thin_flags(m, _ptr(fl), nf, THIN_THRESHOLD, _ptr(a["fwd_thin"]))
    lib.ora_thin_flags(m, _ptr(bl), nb.value, THIN_THRESHOLD, _ptr(a["bck_thin"]))
    a["nnz"] = int(nnz)
    return a


class Oracle:
    """The C restatement over one (matrix, factor) pair."""

    def __init__(self, mat, fac, nt=1, center_k=10, prep=None):
        self.lib = _load_oracle()
        self.n, self.m, self.sddm = mat.n, fac.m, fac.sddm
        self.p = prep if prep is not None else prepare(fac)
        self._keep = [np.ascontiguousarray(mat.colptr, np.int32), np.ascontiguousarray(mat.rowidx, np.int32),
                      np.ascontiguousarray(mat.vals, np.float64), np.ascontiguousarray(fac.perm, np.uint32)]
        a_p, a_i, a_v, perm = self._keep
        p = self.p
        self.s = _System(mat.n, _ptr(a_p), _ptr(a_i), _ptr(a_v), fac.m, int(fac.sddm), _ptr(perm),
                         _ptr(p["csr_ptr"]), _ptr(p["csr_idx"]), _ptr(p["csr_val"]),
                         _ptr(p["csc_ptr"]), _ptr(p["csc_idx"]), _ptr(p["csc_val"]),
                         _ptr(p["fwd_thin"]), _ptr(p["bck_thin"]), nt, center_k, 0)

    def sweep(self, direction, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.m)
        p = self.p
        if direction == 0:
            self.lib.ora_sweep(0, self.m, _ptr(p["csr_ptr"]), _ptr(p["csr_idx"]), _ptr(p["csr_val"]),
                               _ptr(p["fwd_thin"]), _ptr(x), _ptr(y))
        else:
            self.lib.ora_sweep(1, self.m, _ptr(p["csc_ptr"]), _ptr(p["csc_idx"]), _ptr(p["csc_val"]),
                               _ptr(p["bck_thin"]), _ptr(x), _ptr(y))
        return y

    def pair(self, x):
        return self.sweep(1, self.sweep(0, x))

    def apply(self, r, reset=True):
        if reset:
            self.s.apply_count = 0
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.n)
        self.lib.ora_apply(ctypes.byref(self.s), _ptr(r), _ptr(z))
        return z

    def apply_fused(self, r, r_sum, reset=True):
        if reset:
            self.s.apply_count = 0
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.n)
        rz = self.lib.ora_apply_fused(ctypes.byref(self.s), _ptr(r), float(r_sum), _ptr(z))
        return z, rz

    def solve(self, b, tol=1e-8, max_iter=500):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.empty(self.n)
        it = ctypes.c_int(); res = ctypes.c_double()
        self.lib.ora_pcg(ctypes.byref(self.s), _ptr(b), tol, max_iter, _ptr(x), ctypes.byref(it), ctypes.byref(res))
        return x, it.value, res.value
