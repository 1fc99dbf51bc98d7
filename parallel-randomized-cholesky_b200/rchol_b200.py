"""ctypes binding of the C ABI (include/rchol.h) of librchol_b200.so.

This is the Python face of the library for tests, benchmarks and scripting;
it mirrors the reference's host entry points (sparse_matrix_processor,
factorization_driver, prepare_and_solve, the factor write-out).  There is no
CPU fallback: every compute call goes through the sm_100a library and fails
loudly when it or the GPU is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librchol_b200.so")
BIN_DIR = os.path.join(HERE, "bin")

OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "i/o error", 3: "CUDA error", 4: "capacity",
          5: "timeout", 6: "not converged", 7: "no CUDA device", 8: "numeric", 9: "no matrix"}
PREC_FP64, PREC_FP32_FACTOR = 0, 1
STOP_RELRES, STOP_PRECOND, STOP_ABS_R2 = 0, 1, 2
ORDER_GIVEN, ORDER_NNZ_SORT, ORDER_RANDOM, ORDER_RCM, ORDER_ND = 0, 1, 2, 3, 4
SPMV_AUTO, SPMV_CSR = 0, 1

# every symbol include/rchol.h declares
EXPORTS = sorted([
    "rchol_opts_default", "rchol_create", "rchol_destroy", "rchol_set_opts", "rchol_status_string",
    "rchol_last_error", "rchol_load_mtx", "rchol_set_triplets", "rchol_set_csc", "rchol_csc_from_triplets",
    "rchol_read_mtx", "rchol_matrix_info", "rchol_matrix_copy_to_host", "rchol_factor", "rchol_factor_get_info",
    "rchol_factor_copy_to_host", "rchol_factor_write", "rchol_factor_read", "rchol_factor_from_csr_upper",
    "rchol_factor_free", "rchol_pcg_solve", "rchol_precond_apply", "rchol_precond_apply_noalloc", "rchol_profile_solve", "rchol_spmv", "rchol_factorization_driver",
    "rchol_prepare_and_solve", "rchol_generate", "rchol_free_host", "rchol_write_mtx", "rchol_batch_set",
    "rchol_batch_solve", "rchol_zero_sum_vector", "rchol_set_sddm", "rchol_write_bin", "rchol_read_bin",
    "rchol_save_bin", "rchol_load_bin", "rchol_autotune", "rchol_ordering",
    "rchol_hop_latency",
])


class RcholError(RuntimeError):
    def __init__(self, status, msg=""):
        super().__init__(f"rchol: {STATUS.get(status, status)}" + (f": {msg}" if msg else ""))
        self.status = status


class Opts(C.Structure):
    _fields_ = [("precision", C.c_int), ("seed", C.c_ulonglong), ("num_blocks", C.c_int),
                ("warps_per_block", C.c_int), ("slab_entries", C.c_int), ("bucket_cap", C.c_int),
                ("pool_mult", C.c_double), ("max_iter", C.c_int), ("tol", C.c_double), ("stop_rule", C.c_int),
                ("unroll", C.c_int), ("use_graph", C.c_int), ("device", C.c_int), ("timeout_s", C.c_double),
                ("verbose", C.c_int), ("poll_ns", C.c_int),
                ("sched_epl", C.c_int), ("exact_bwd_levels", C.c_int), ("spmv_layout", C.c_int),
                ("tail_vertices", C.c_int), ("rhs_block", C.c_int), ("bwd_head", C.c_int)]


class FactorInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("n_factored", C.c_int), ("nnz_strict", C.c_longlong),
                ("nnz_lower_a", C.c_longlong), ("fills", C.c_longlong), ("max_gather", C.c_int),
                ("big_vertices", C.c_int), ("overflow_fills", C.c_int), ("chunks_used", C.c_int),
                ("factor_grid", C.c_int), ("ms_setup", C.c_float), ("ms_factor", C.c_float),
                ("ms_assemble", C.c_float), ("attempts", C.c_int),
                ("solve_depth", C.c_int), ("kernel_launches", C.c_int),
                ("lc_ptr", C.c_void_p), ("lc_idx", C.c_void_p), ("lc_val", C.c_void_p),
                ("lr_ptr", C.c_void_p), ("lr_idx", C.c_void_p), ("lr_val", C.c_void_p), ("diag", C.c_void_p),
                ("tail_vertices", C.c_int), ("solve_depth_b", C.c_int), ("bwd_head_levels", C.c_int),
                ("bwd_head_rows", C.c_int)]


class TuneResult(C.Structure):
    _fields_ = [("tail_vertices", C.c_int), ("bucket_cap", C.c_int), ("rhs_block", C.c_int),
                ("from_cache", C.c_int), ("max_gather", C.c_int), ("ms_factor_default", C.c_float),
                ("ms_factor_tuned", C.c_float), ("per_rhs_ms", C.c_float * 6)]


class System(C.Structure):
    _fields_ = [("n", C.c_int), ("colptr", C.c_void_p), ("rowind", C.c_void_p), ("val", C.c_void_p)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("device_status", C.c_int),
                ("relres_true", C.c_double), ("relres_rec", C.c_double), ("precond_ratio", C.c_double),
                ("ms_total", C.c_float), ("ms_iterations", C.c_float), ("kernel_launches", C.c_int),
                ("graph_launches", C.c_int)]


def _struct_dict(s):
    return {k: getattr(s, k) for k, _ in s._fields_ if not k.endswith(("_ptr", "_idx", "_val")) and k != "diag"}


_lib = None


def build(force=False):
    """Compile the library and drivers in-tree (nvcc, sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RcholError(3, f"{LIB_PATH} is not built (run make -C {HERE})")
        L = C.CDLL(LIB_PATH)
        vp, i32p, i64p, f64p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_double)
        L.rchol_opts_default.argtypes = [C.POINTER(Opts)]
        L.rchol_create.argtypes = [C.POINTER(vp), C.POINTER(Opts)]
        L.rchol_destroy.argtypes = [vp]
        L.rchol_destroy.restype = None
        L.rchol_set_opts.argtypes = [vp, C.POINTER(Opts)]
        L.rchol_status_string.restype = C.c_char_p
        L.rchol_last_error.argtypes = [vp]
        L.rchol_last_error.restype = C.c_char_p
        L.rchol_load_mtx.argtypes = [vp, C.c_char_p, C.c_int]
        L.rchol_set_triplets.argtypes = [vp, C.c_int, C.c_longlong, vp, vp, vp, C.c_int]
        L.rchol_set_csc.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, C.c_int]
        L.rchol_csc_from_triplets.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, vp, vp, vp, i64p]
        L.rchol_read_mtx.argtypes = [C.c_char_p, i32p, i64p, C.POINTER(i32p), C.POINTER(i32p), C.POINTER(f64p)]
        L.rchol_matrix_info.argtypes = [vp, i32p, i64p]
        L.rchol_matrix_copy_to_host.argtypes = [vp, vp, vp, vp]
        L.rchol_factor.argtypes = [vp, C.POINTER(vp)]
        L.rchol_factor_get_info.argtypes = [vp, C.POINTER(FactorInfo)]
        L.rchol_factor_copy_to_host.argtypes = [vp, vp, vp, vp, vp]
        L.rchol_factor_write.argtypes = [vp, C.c_char_p]
        L.rchol_factor_read.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
        L.rchol_factor_from_csr_upper.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_int, C.POINTER(vp)]
        L.rchol_factor_free.argtypes = [vp]
        L.rchol_factor_free.restype = None
        L.rchol_pcg_solve.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, C.POINTER(SolveInfo)]
        L.rchol_precond_apply.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, C.c_int]
        L.rchol_precond_apply_noalloc.argtypes = [vp, C.c_int, vp, vp, C.c_int, vp]
        L.rchol_spmv.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.c_int]
        L.rchol_profile_solve.argtypes = [vp, vp, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.rchol_hop_latency.argtypes = [vp, C.c_int, C.POINTER(C.c_double), i32p]
        L.rchol_factorization_driver.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_int]
        L.rchol_prepare_and_solve.argtypes = [C.c_int, C.c_longlong, vp, vp, vp, vp, vp, vp, vp, C.c_double,
                                              C.c_int, C.c_longlong, C.c_int, vp, C.POINTER(SolveInfo)]
        L.rchol_generate.argtypes = [C.c_char_p, C.POINTER(C.c_longlong), C.c_int, C.c_double, C.c_double,
                                     C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                     C.c_ulonglong, i32p, i64p, C.POINTER(i32p), C.POINTER(i32p),
                                     C.POINTER(f64p), i32p]
        L.rchol_free_host.argtypes = [vp]
        L.rchol_free_host.restype = None
        L.rchol_write_mtx.argtypes = [C.c_char_p, C.c_int, C.c_longlong, vp, vp, vp]
        L.rchol_zero_sum_vector.argtypes = [C.c_int, C.c_uint, vp]
        L.rchol_write_bin.argtypes = [C.c_char_p, C.c_int, vp, vp, vp, C.c_int]
        L.rchol_read_bin.argtypes = [C.c_char_p, i32p, i64p, C.POINTER(i32p), C.POINTER(i32p), C.POINTER(f64p),
                                     i32p]
        L.rchol_save_bin.argtypes = [vp, C.c_char_p]
        L.rchol_load_bin.argtypes = [vp, C.c_char_p]
        L.rchol_autotune.argtypes = [vp, C.c_int, C.POINTER(TuneResult)]
        L.rchol_ordering.argtypes = [C.c_int, C.c_int, C.c_longlong, vp, vp, vp]
        L.rchol_set_sddm.argtypes = [vp, C.c_int, C.c_longlong, vp, vp, vp, C.c_int, C.c_int, C.c_ulonglong, vp,
                                     i32p]
        L.rchol_batch_set.argtypes = [vp, C.c_int, C.POINTER(System), C.POINTER(C.c_longlong)]
        L.rchol_batch_solve.argtypes = [vp, vp, C.c_int, vp, vp, C.c_int, C.c_int, C.POINTER(SolveInfo),
                                        C.POINTER(SolveInfo)]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def _check(st, ctx=None):
    if st != OK:
        msg = ""
        if ctx:
            msg = (lib().rchol_last_error(ctx) or b"").decode()
        raise RcholError(st, msg)


def default_opts(**kw):
    o = Opts()
    lib().rchol_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


# ---------------------------------------------------------------------------
# host-only helpers (no GPU needed)
# ---------------------------------------------------------------------------

def generate(kind, dims, wlo=1.0, whi=1.0, log_weights=False, aniso_z=1.0, excess_frac=0.0, excess_lo=0.0,
             excess_hi=0.0, ordering=0, seed=0):
    """Synthetic Laplacian triplets (see rchol_generate)."""
    L = lib()
    d = (C.c_longlong * len(dims))(*dims)
    n = C.c_int()
    nnz = C.c_longlong()
    r = C.POINTER(C.c_int)()
    c = C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    g = C.c_int()
    st = L.rchol_generate(kind.encode(), d, len(dims), wlo, whi, int(log_weights), aniso_z, excess_frac,
                          excess_lo, excess_hi, ordering, seed, C.byref(n), C.byref(nnz), C.byref(r), C.byref(c),
                          C.byref(v), C.byref(g))
    _check(st)
    m = nnz.value
    rows = np.ctypeslib.as_array(r, shape=(m,)).copy()
    cols = np.ctypeslib.as_array(c, shape=(m,)).copy()
    vals = np.ctypeslib.as_array(v, shape=(m,)).copy()
    for p in (r, c, v):
        L.rchol_free_host(C.cast(p, C.c_void_p))
    return n.value, rows, cols, vals, bool(g.value)


def csc_from_triplets(n, rows, cols, vals):
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    nnz = C.c_longlong()
    _check(lib().rchol_csc_from_triplets(n, len(rows), _ptr(rows), _ptr(cols), _ptr(vals), None, None, None,
                                         C.byref(nnz)))
    colptr = np.zeros(n + 1, np.int32)
    rowind = np.zeros(max(nnz.value, 1), np.int32)
    val = np.zeros(max(nnz.value, 1), np.float64)
    _check(lib().rchol_csc_from_triplets(n, len(rows), _ptr(rows), _ptr(cols), _ptr(vals), _ptr(colptr),
                                         _ptr(rowind), _ptr(val), C.byref(nnz)))
    return colptr, rowind[:nnz.value], val[:nnz.value]


def read_mtx(path):
    L = lib()
    n = C.c_int()
    nnz = C.c_longlong()
    r = C.POINTER(C.c_int)()
    c = C.POINTER(C.c_int)()
    v = C.POINTER(C.c_double)()
    _check(L.rchol_read_mtx(path.encode(), C.byref(n), C.byref(nnz), C.byref(r), C.byref(c), C.byref(v)))
    m = nnz.value
    out = (n.value, np.ctypeslib.as_array(r, shape=(m,)).copy(), np.ctypeslib.as_array(c, shape=(m,)).copy(),
           np.ctypeslib.as_array(v, shape=(m,)).copy())
    for p in (r, c, v):
        L.rchol_free_host(C.cast(p, C.c_void_p))
    return out


def write_bin(path, n, colptr, rowind, val, trim_ground=False):
    """Binary matrix cache of a preprocessed CSC (rchol_write_bin)."""
    colptr = np.ascontiguousarray(colptr, np.int32)
    rowind = np.ascontiguousarray(rowind, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    _check(lib().rchol_write_bin(path.encode(), n, _ptr(colptr), _ptr(rowind), _ptr(val), int(trim_ground)))


def read_bin(path):
    """(n, colptr, rowind, val, trim_ground) of a binary matrix cache."""
    L = lib()
    n, nnz, tr = C.c_int(), C.c_longlong(), C.c_int()
    cp, ri, v = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    _check(L.rchol_read_bin(path.encode(), C.byref(n), C.byref(nnz), C.byref(cp), C.byref(ri), C.byref(v),
                            C.byref(tr)))
    try:
        out = (n.value, np.ctypeslib.as_array(cp, (n.value + 1,)).copy(),
               np.ctypeslib.as_array(ri, (max(nnz.value, 1),))[:nnz.value].copy(),
               np.ctypeslib.as_array(v, (max(nnz.value, 1),))[:nnz.value].copy(), bool(tr.value))
    finally:
        for p in (cp, ri, v):
            L.rchol_free_host(C.cast(p, C.c_void_p))
    return out


def ordering(kind, n, rows, cols):
    """Host RCM (ORDER_RCM) or nested-dissection (ORDER_ND) order of a
    symmetric pattern: order[k] = vertex placed at position k."""
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    out = np.zeros(n, np.int32)
    _check(lib().rchol_ordering(int(kind), int(n), len(rows), _ptr(rows), _ptr(cols), _ptr(out)))
    return out


def zero_sum_vector(n, seed=0):
    """The reference right-hand side generate_zero_sum_vector(n, seed)
    (gpu_implementation/solver.hpp:43-61), host only."""
    out = np.zeros(n, np.float64)
    _check(lib().rchol_zero_sum_vector(int(n), int(seed), _ptr(out)))
    return out


def write_mtx(path, n, rows, cols, vals):
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    _check(lib().rchol_write_mtx(path.encode(), n, len(rows), _ptr(rows), _ptr(cols), _ptr(vals)))


# ---------------------------------------------------------------------------
# context / factor
# ---------------------------------------------------------------------------

class Factor:
    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    def info(self):
        fi = FactorInfo()
        _check(lib().rchol_factor_get_info(self.h, C.byref(fi)))
        return fi

    def to_host(self):
        """Strict CSC of L (rows ascending, values L_ij) and D."""
        fi = self.info()
        n, nnz = fi.n, fi.nnz_strict
        colptr = np.zeros(n + 1, np.int64)
        rowind = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1), np.float64)
        diag = np.zeros(max(n, 1), np.float64)
        _check(lib().rchol_factor_copy_to_host(self.h, _ptr(colptr), _ptr(rowind), _ptr(val), _ptr(diag)),
               self.ctx.h)
        return colptr, rowind[:nnz], val[:nnz], diag[:n]

    def write(self, prefix):
        _check(lib().rchol_factor_write(self.h, prefix.encode()), self.ctx.h)

    def free(self):
        if self.h:
            lib().rchol_factor_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Context:
    def __init__(self, opts=None, **kw):
        self.h = C.c_void_p()
        o = opts if opts is not None else default_opts(**kw)
        _check(lib().rchol_create(C.byref(self.h), C.byref(o)))
        self.opts = o

    def close(self):
        if self.h:
            lib().rchol_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_opts(self, **kw):
        for k, v in kw.items():
            setattr(self.opts, k, v)
        _check(lib().rchol_set_opts(self.h, C.byref(self.opts)), self.h)

    def load_mtx(self, path, trim_ground=False):
        _check(lib().rchol_load_mtx(self.h, path.encode(), int(trim_ground)), self.h)

    def set_triplets(self, n, rows, cols, vals, trim_ground=False):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        _check(lib().rchol_set_triplets(self.h, n, len(rows), _ptr(rows), _ptr(cols), _ptr(vals),
                                        int(trim_ground)), self.h)

    def set_sddm(self, n, rows, cols, vals, ordering=ORDER_NNZ_SORT, order_seed=0):
        """An SDDM or Laplacian converted and ordered on the device
        (rchol_set_sddm).  Returns (perm, has_ground): perm[i] = position of
        input vertex i in the context's matrix."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        perm = np.zeros(n, np.int32)
        g = C.c_int(0)
        _check(lib().rchol_set_sddm(self.h, n, len(rows), _ptr(rows), _ptr(cols), _ptr(vals), 0, int(ordering),
                                    int(order_seed), _ptr(perm), C.byref(g)), self.h)
        return perm, bool(g.value)

    def autotune(self, max_rhs=1):
        """rchol_autotune: the chosen options (also set on the context)."""
        r = TuneResult()
        _check(lib().rchol_autotune(self.h, int(max_rhs), C.byref(r)), self.h)
        d = {k: getattr(r, k) for k, _ in r._fields_ if k != "per_rhs_ms"}
        d["per_rhs_ms"] = list(r.per_rhs_ms)
        # the context now runs with the tuned options; keep this copy in step
        for k in ("tail_vertices", "bucket_cap", "rhs_block"):
            setattr(self.opts, k, d[k])
        return d

    def load_bin(self, path):
        _check(lib().rchol_load_bin(self.h, path.encode()), self.h)

    def save_bin(self, path):
        _check(lib().rchol_save_bin(self.h, path.encode()), self.h)

    def set_csc(self, n, colptr, rowind, val, trim_ground=False, on_device=False):
        if on_device:
            _check(lib().rchol_set_csc(self.h, n, C.c_void_p(colptr), C.c_void_p(rowind), C.c_void_p(val), 1,
                                       int(trim_ground)), self.h)
            return
        colptr = np.ascontiguousarray(colptr, np.int32)
        rowind = np.ascontiguousarray(rowind, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        _check(lib().rchol_set_csc(self.h, n, _ptr(colptr), _ptr(rowind), _ptr(val), 0, int(trim_ground)),
               self.h)

    def matrix(self):
        n = C.c_int()
        nnz = C.c_longlong()
        _check(lib().rchol_matrix_info(self.h, C.byref(n), C.byref(nnz)), self.h)
        colptr = np.zeros(n.value + 1, np.int32)
        rowind = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value, np.float64)
        _check(lib().rchol_matrix_copy_to_host(self.h, _ptr(colptr), _ptr(rowind), _ptr(val)), self.h)
        return n.value, colptr, rowind, val

    def factor(self):
        h = C.c_void_p()
        _check(lib().rchol_factor(self.h, C.byref(h)), self.h)
        return Factor(self, h)

    def factor_read(self, prefix):
        h = C.c_void_p()
        _check(lib().rchol_factor_read(self.h, prefix.encode(), C.byref(h)), self.h)
        return Factor(self, h)

    def factor_from_csr_upper(self, n, rowptr, colind, val, diag):
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        colind = np.ascontiguousarray(colind, np.int32)
        val = np.ascontiguousarray(val, np.float64)
        diag = np.ascontiguousarray(diag, np.float64)
        h = C.c_void_p()
        _check(lib().rchol_factor_from_csr_upper(self.h, n, _ptr(rowptr), _ptr(colind), _ptr(val), _ptr(diag), 0,
                                                 C.byref(h)), self.h)
        return Factor(self, h)

    def pcg_solve(self, factor, B, raise_on_nonconv=False):
        """Solve A X = B; B is (n,) or (n, k) (column-major copy made)."""
        B = np.asarray(B, np.float64)
        vec = B.ndim == 1
        Bm = B.reshape(-1, 1) if vec else B
        n, k = Bm.shape
        Bf = np.asfortranarray(Bm)
        X = np.zeros((n, k), np.float64, order="F")
        si = SolveInfo()
        st = lib().rchol_pcg_solve(self.h, factor.h, k, Bf.ctypes.data_as(C.c_void_p), X.ctypes.data_as(C.c_void_p),
                                   n, 0, C.byref(si))
        if st not in (OK, 6) or (st == 6 and raise_on_nonconv):
            _check(st, self.h)
        info = _struct_dict(si)
        info["status"] = st
        return (X[:, 0].copy() if vec else np.ascontiguousarray(X)), info

    def pcg_solve_device(self, factor, k, b_ptr, x_ptr, ldb):
        """Device-resident B/X (column-major, leading dimension ldb)."""
        si = SolveInfo()
        st = lib().rchol_pcg_solve(self.h, factor.h, k, C.c_void_p(b_ptr), C.c_void_p(x_ptr), ldb, 1, C.byref(si))
        if st not in (OK, 6):
            _check(st, self.h)
        info = _struct_dict(si)
        info["status"] = st
        return info

    def precond_apply(self, factor, R, fp32=False):
        R = np.asarray(R, np.float64)
        vec = R.ndim == 1
        Rm = R.reshape(-1, 1) if vec else R
        n, k = Rm.shape
        Rf = np.asfortranarray(Rm)
        Z = np.zeros((n, k), np.float64, order="F")
        _check(lib().rchol_precond_apply(self.h, factor.h, k, Rf.ctypes.data_as(C.c_void_p),
                                         Z.ctypes.data_as(C.c_void_p), n, 0, int(fp32)), self.h)
        return Z[:, 0].copy() if vec else np.ascontiguousarray(Z)

    def precond_apply_noalloc(self, factor, r_ptr, z_ptr, k=1, fp32=False, stream=0):
        """Z = M^+ R on caller-owned device arrays (row-major n x k, given as
        integer device addresses) without any device allocation; scratch is
        a fixed library array (n * k <= 2**22), shared by every call on the
        device, so overlapping calls must be serialised by the caller."""
        _check(lib().rchol_precond_apply_noalloc(factor.h, int(k), C.c_void_p(r_ptr), C.c_void_p(z_ptr), int(fp32),
                                                 C.c_void_p(stream or None)), self.h)

    def batch_set(self, systems):
        """systems: list of (n, colptr, rowind, val) preprocessed CSC arrays.
        Returns the row offsets of the block-diagonal stacking."""
        keep = []
        arr = (System * len(systems))()
        for q, (n, cp, ri, v) in enumerate(systems):
            cp = np.ascontiguousarray(cp, np.int32)
            ri = np.ascontiguousarray(ri, np.int32)
            v = np.ascontiguousarray(v, np.float64)
            keep += [cp, ri, v]
            arr[q] = System(n, _ptr(cp), _ptr(ri), _ptr(v))
        off = (C.c_longlong * (len(systems) + 1))()
        _check(lib().rchol_batch_set(self.h, len(systems), arr, off), self.h)
        self.batch_offsets = np.array(off[:], np.int64)
        return self.batch_offsets

    def batch_solve(self, factor, B):
        """B: (n_total,) or (n_total, k); returns X, per-system info, total info."""
        B = np.asarray(B, np.float64)
        vec = B.ndim == 1
        Bm = B.reshape(-1, 1) if vec else B
        n, k = Bm.shape
        Bf = np.asfortranarray(Bm)
        X = np.zeros((n, k), np.float64, order="F")
        nsys = len(self.batch_offsets) - 1
        per = (SolveInfo * nsys)()
        tot = SolveInfo()
        st = lib().rchol_batch_solve(self.h, factor.h, k, Bf.ctypes.data_as(C.c_void_p),
                                     X.ctypes.data_as(C.c_void_p), n, 0, per, C.byref(tot))
        if st not in (OK, 6):
            _check(st, self.h)
        info = _struct_dict(tot)
        info["status"] = st
        return (X[:, 0].copy() if vec else np.ascontiguousarray(X)), [_struct_dict(p) for p in per], info

    def profile_solve(self, factor, k=1, reps=5):
        """Mean ms of (spmv_update, fwd, bwd) per iteration."""
        ms = (C.c_float * 3)()
        _check(lib().rchol_profile_solve(self.h, factor.h, k, reps, ms), self.h)
        return list(ms)

    def hop_latency(self, rounds=4096):
        """(ns per store -> poll hop between two SMs, (sm_a, sm_b)): the latency
        floor per level of the sync-free triangular solves."""
        ns = C.c_double()
        sm = (C.c_int * 2)()
        _check(lib().rchol_hop_latency(self.h, rounds, C.byref(ns), sm), self.h)
        return ns.value, (sm[0], sm[1])

    def spmv(self, X):
        X = np.asarray(X, np.float64)
        vec = X.ndim == 1
        Xm = X.reshape(-1, 1) if vec else X
        n, k = Xm.shape
        Xf = np.asfortranarray(Xm)
        Y = np.zeros((n, k), np.float64, order="F")
        _check(lib().rchol_spmv(self.h, k, Xf.ctypes.data_as(C.c_void_p), Y.ctypes.data_as(C.c_void_p), n, 0),
               self.h)
        return Y[:, 0].copy() if vec else np.ascontiguousarray(Y)


def prepare_and_solve(lap_n, lap_rowptr, lap_colind, lap_val, csr_rowptr, csr_val, csr_colind, diag, tol,
                      physics=True, removal=False, x_out=0):
    """solver.hpp:236 drop-in on device pointers (ints)."""
    si = SolveInfo()
    st = lib().rchol_prepare_and_solve(lap_n, 0, C.c_void_p(lap_rowptr), C.c_void_p(lap_colind),
                                       C.c_void_p(lap_val), C.c_void_p(csr_rowptr), C.c_void_p(csr_val),
                                       C.c_void_p(csr_colind), C.c_void_p(diag), tol, int(physics), 0,
                                       int(removal), C.c_void_p(x_out) if x_out else None, C.byref(si))
    _check(st)
    return _struct_dict(si)


def driver_binary(name):
    return os.path.join(BIN_DIR, name)
