"""ctypes access to the C oracle (liboracle.so) and to the reference CPU factor
built under oracle/_ref/.  Test infrastructure: imported only by tests/,
__graft_entry__.smoke() and the CPU-baseline leg of bench.py.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "rchol_ref_cpu")
REF_BIN_PINNED = os.path.join(HERE, "_ref", "rchol_ref_cpu_pinned")

MODE_B200 = 0
MODE_REF_REPLAY = 1
STOP_RELRES = 0
STOP_PRECOND = 1
STOP_ABS_R2 = 2

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


class FactorStats(C.Structure):
    _fields_ = [("nnz_strict", C.c_int64), ("fills", C.c_int64), ("merged_away", C.c_int64),
                ("max_degree", C.c_int32), ("max_gather", C.c_int32)]


class PcgInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("relres_true", C.c_double),
                ("relres_rec", C.c_double), ("precond_ratio", C.c_double)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_zero_sum_vector.argtypes = [_f64p, C.c_int64, C.c_uint32]
        L.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
        L.orc_sample_uniform.argtypes = [C.c_uint64, C.c_int32, C.c_int32]
        L.orc_sample_uniform.restype = C.c_double
        L.orc_has_diagonal.argtypes = [C.c_int64, _i32p, _i32p]
        L.orc_triplets_to_csc.argtypes = [C.c_int32, C.c_int64, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.orc_triplets_to_csc.restype = C.c_int64
        L.orc_lower_count.argtypes = [C.c_int32, _i32p, _i32p]
        L.orc_lower_count.restype = C.c_int64
        L.orc_lower_triangle.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.orc_dependency_counts.argtypes = [C.c_int32, _i32p, _i32p, _i32p]
        L.orc_trim_last.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        L.orc_trim_last.restype = C.c_int64
        L.orc_factor_run.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _i32p, C.c_int, C.c_uint64]
        L.orc_factor_run.restype = C.c_void_p
        L.orc_factor_stats_get.argtypes = [C.c_void_p, C.POINTER(FactorStats)]
        L.orc_factor_export.argtypes = [C.c_void_p, _i64p, _i32p, _f64p, _f64p, _i32p]
        L.orc_factor_free.argtypes = [C.c_void_p]
        L.orc_spmv.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int]
        L.orc_precond_apply.argtypes = [C.c_int32, _i64p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p]
        L.orc_pcg.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _i64p, _i32p, _f64p, _f64p,
                              _f64p, _f64p, C.c_double, C.c_int32, C.c_int, C.c_int,
                              C.POINTER(PcgInfo)]
        L.orc_pcg.restype = C.c_int
        L.orc_generate_grid.argtypes = [C.c_char_p, _i64p, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double,
                                        C.c_double, C.c_double, C.c_double, C.c_uint64, C.POINTER(C.c_int32),
                                        C.POINTER(C.c_int64), C.POINTER(C.POINTER(C.c_int32)),
                                        C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_double)),
                                        C.POINTER(C.c_int32)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_free.restype = None
        L.orc_write_mtx.argtypes = [C.c_char_p, C.c_int32, C.c_int64, _i32p, _i32p, _f64p]
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def zero_sum_vector(n, seed=0):
    out = np.empty(n, np.float64)
    lib().orc_zero_sum_vector(out, n, seed)
    return out


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def sample_uniform(seed, vertex, i):
    return lib().orc_sample_uniform(seed, vertex, i)


def triplets_to_csc(n, rows, cols, vals):
    rows, cols, vals = _i32(rows), _i32(cols), _f64(vals)
    has_diag = lib().orc_has_diagonal(len(rows), rows, cols)
    total = len(rows) + (0 if has_diag else n)
    colptr = np.zeros(n + 1, np.int32)
    rowind = np.zeros(max(total, 1), np.int32)
    val = np.zeros(max(total, 1), np.float64)
    got = lib().orc_triplets_to_csc(n, len(rows), rows, cols, vals, colptr, rowind, val)
    return colptr, rowind[:got], val[:got]


def lower_triangle(n, colptr, rowind, val):
    colptr, rowind, val = _i32(colptr), _i32(rowind), _f64(val)
    cnt = lib().orc_lower_count(n, colptr, rowind)
    lcp = np.zeros(n + 1, np.int32)
    lr = np.zeros(max(cnt, 1), np.int32)
    lv = np.zeros(max(cnt, 1), np.float64)
    lib().orc_lower_triangle(n, colptr, rowind, val, lcp, lr, lv)
    return lcp, lr[:cnt], lv[:cnt]


def dependency_counts(n, colptr, rowind):
    dep = np.zeros(n, np.int32)
    lib().orc_dependency_counts(n, _i32(colptr), _i32(rowind), dep)
    return dep


def trim_last(n, colptr, rowind, val):
    colptr, rowind, val = _i32(colptr), _i32(rowind), _f64(val)
    ocp = np.zeros(n, np.int32)
    orow = np.zeros(max(len(rowind), 1), np.int32)
    oval = np.zeros(max(len(rowind), 1), np.float64)
    got = lib().orc_trim_last(n, colptr, rowind, val, ocp, orow, oval)
    return ocp, orow[:got], oval[:got]


def factor(n, lcolptr, lrow, lval, dep0, mode=MODE_B200, seed=1):
    L = lib()
    h = L.orc_factor_run(n, _i32(lcolptr), _i32(lrow), _f64(lval), _i32(dep0), mode, seed)
    if not h:
        raise MemoryError("oracle factor failed")
    st = FactorStats()
    L.orc_factor_stats_get(h, C.byref(st))
    nnz = st.nnz_strict
    colptr = np.zeros(n + 1, np.int64)
    rowind = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), np.float64)
    diag = np.zeros(max(n, 1), np.float64)
    fills = np.zeros(max(n, 1), np.int32)
    L.orc_factor_export(h, colptr, rowind, val, diag, fills)
    L.orc_factor_free(h)
    return dict(colptr=colptr, rowind=rowind[:nnz], val=val[:nnz], diag=diag[:n],
                fills_received=fills[:n],
                stats=dict(nnz_strict=st.nnz_strict, fills=st.fills, merged_away=st.merged_away,
                           max_degree=st.max_degree, max_gather=st.max_gather))


def spmv(n, rowptr, colind, val, x, nthreads=1):
    y = np.zeros(n, np.float64)
    lib().orc_spmv(n, _i32(rowptr), _i32(colind), _f64(val), _f64(x), y, nthreads)
    return y


def precond_apply(n, lcolptr, lrow, lval, diag, r):
    z = np.zeros(n, np.float64)
    work = np.zeros(n, np.float64)
    lib().orc_precond_apply(n, np.ascontiguousarray(lcolptr, np.int64), _i32(lrow), _f64(lval),
                            _f64(diag), _f64(r), z, work)
    return z


def pcg(n, arowptr, acolind, aval, lcolptr, lrow, lval, diag, b, tol=1e-6, max_iter=1000,
        stop_rule=STOP_RELRES, nthreads=1):
    x = np.zeros(n, np.float64)
    info = PcgInfo()
    rc = lib().orc_pcg(n, _i32(arowptr), _i32(acolind), _f64(aval),
                       np.ascontiguousarray(lcolptr, np.int64), _i32(lrow), _f64(lval),
                       _f64(diag), _f64(b), x, tol, max_iter, stop_rule, nthreads, C.byref(info))
    if rc != 0:
        raise MemoryError("oracle pcg failed")
    return x, dict(iterations=info.iterations, converged=bool(info.converged),
                   relres_true=info.relres_true, relres_rec=info.relres_rec,
                   precond_ratio=info.precond_ratio)


def generate_grid(kind, dims, wlo=1.0, whi=1.0, log_weights=False, aniso_z=1.0, excess_frac=0.0, excess_lo=0.0,
                  excess_hi=0.0, seed=0):
    """The benchmark grid inputs (same triplets as the library's generator)
    built by oracle/gen_inputs.c: (n, rows, cols, vals, has_ground)."""
    L = lib()
    d = np.ascontiguousarray(dims, np.int64)
    n, nnz, g = C.c_int32(), C.c_int64(), C.c_int32()
    rp, cp, vp = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), C.POINTER(C.c_double)()
    rc = L.orc_generate_grid(kind.encode(), d, len(d), wlo, whi, int(log_weights), aniso_z, excess_frac, excess_lo,
                             excess_hi, seed, C.byref(n), C.byref(nnz), C.byref(rp), C.byref(cp), C.byref(vp),
                             C.byref(g))
    if rc != 0:
        raise ValueError(f"orc_generate_grid failed ({rc})")
    m = nnz.value
    try:
        rows = np.ctypeslib.as_array(rp, (m,)).copy()
        cols = np.ctypeslib.as_array(cp, (m,)).copy()
        vals = np.ctypeslib.as_array(vp, (m,)).copy()
    finally:
        L.orc_free(C.cast(rp, C.c_void_p))
        L.orc_free(C.cast(cp, C.c_void_p))
        L.orc_free(C.cast(vp, C.c_void_p))
    return n.value, rows, cols, vals, bool(g.value)


_M64 = (1 << 64) - 1


def _mix64(x):
    """splitmix64 finaliser on numpy uint64 arrays (wrapping arithmetic)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def order_keys(n, seed):
    """The 64-bit ordering key of every vertex: splitmix64 of (seed,
    stream 4, vertex), the tie-break of the ascending-nnz order."""
    with np.errstate(over="ignore"):
        base = _mix64(_mix64(np.array([seed], np.uint64)) ^ np.uint64((4 * 0xD1B54A32D192ED03) & _M64))
        return _mix64(base ^ np.arange(n, dtype=np.uint64))


def sddm_to_laplacian(n, rows, cols, vals, ordering=1, seed=0, order=None):
    """Restatement of the physics preprocessing (cpu_implementation/
    write_graph.jl:98-183) as rchol_set_sddm performs it: sign
    normalisation (and a diagonal of sum |off| per column when the input has
    none), the ordering (0 given, 1 ascending column nnz after the seeded
    permutation, 2 the seeded permutation, or an explicit `order`), and the
    ground vertex appended
    when the entries sum to more than 1e-9.  Column sums are added in row
    order, the ground diagonal in column order.  Returns
    (N, colptr, rowind, val, perm, has_ground).  Small inputs only."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    vals = np.asarray(vals, np.float64)
    v = np.where(rows == cols, np.abs(vals), -np.abs(vals))
    append_diag = not np.any(rows == cols)
    cnt = np.bincount(cols, minlength=n)
    ident = np.arange(n)
    if order is not None:  # an order computed elsewhere (RCM, nested dissection)
        order = np.asarray(order, np.int64)
    elif ordering == 0:
        order = ident
    else:
        key = order_keys(n, seed)
        order = np.lexsort((ident, key, cnt)) if ordering == 1 else np.lexsort((ident, key))
    pos = np.empty(n, np.int64)
    pos[order] = ident
    pr, pc = pos[rows], pos[cols]
    if append_diag:
        pr = np.concatenate([pr, pos])
        pc = np.concatenate([pc, pos])
        v = np.concatenate([v, np.zeros(n)])
    e = np.lexsort((np.arange(len(pr)), pr, pc))
    ri, cc, val = pr[e], pc[e], v[e].copy()
    cp = np.concatenate([[0], np.cumsum(np.bincount(cc, minlength=n))])
    if append_diag:
        for j in range(n):
            s_ = 0.0
            d = -1
            for p in range(cp[j], cp[j + 1]):
                if ri[p] == j:
                    d = p
                else:
                    s_ += abs(val[p])
            if d >= 0:
                val[d] = s_
    csum = np.zeros(n)
    pos_c = np.zeros(n, bool)
    for j in range(n):
        s_ = 0.0
        a_ = 0.0
        for p in range(cp[j], cp[j + 1]):
            s_ += val[p]
            a_ += abs(val[p])
        csum[j] = s_
        # a column sum within the rounding bound of its own sum counts as zero
        pos_c[j] = s_ > float(cp[j + 1] - cp[j]) * 2.0 ** -52 * a_
    total = float(np.sum(csum))
    if total < -1e-9:
        raise ValueError("not diagonally dominant")
    if not total > 1e-9:
        return n, cp.astype(np.int32), ri.astype(np.int32), val, pos.astype(np.int32), False
    g = np.nonzero(pos_c)[0]
    gd = 0.0
    for j in g:
        gd += csum[j]
    ncp = [0]
    nri, nval = [], []
    for j in range(n):
        nri.append(ri[cp[j]:cp[j + 1]])
        nval.append(val[cp[j]:cp[j + 1]])
        if pos_c[j]:
            nri.append(np.array([n]))
            nval.append(np.array([-csum[j]]))
        ncp.append(ncp[-1] + (cp[j + 1] - cp[j]) + (1 if pos_c[j] else 0))
    nri.append(g)
    nval.append(-csum[g])
    nri.append(np.array([n]))
    nval.append(np.array([gd]))
    ncp.append(ncp[-1] + len(g) + 1)
    return (n + 1, np.array(ncp, np.int32), np.concatenate(nri).astype(np.int32), np.concatenate(nval),
            pos.astype(np.int32), True)


def write_mtx_fast(path, n, rows, cols, vals):
    """write_mtx in C (large inputs)."""
    if lib().orc_write_mtx(path.encode(), n, len(rows), _i32(rows), _i32(cols), _f64(vals)) != 0:
        raise OSError(f"could not write {path}")


# ---------------------------------------------------------------------------
# MatrixMarket text IO (small test inputs) and the reference CPU factor
# ---------------------------------------------------------------------------

def write_mtx(path, n, rows, cols, vals):
    """1-based coordinate/real/general file, entries in the given order."""
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(rows)}\n")
        lines = [f"{r + 1} {c + 1} {v:.17g}\n" for r, c, v in zip(rows, cols, vals)]
        f.write("".join(lines))


def read_factor_files(prefix, n):
    """Read <prefix>l_sol.mtx (1-based CSC of L incl. unit diagonal) and
    <prefix>sol_diag.txt as written by driver_local.cpp:958-988."""
    with open(prefix + "l_sol.mtx") as f:
        header = f.readline()
        assert header.startswith("%%MatrixMarket")
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nnz = map(int, line.split())
        if nnz == 0:
            data = np.zeros((0, 3))
        else:
            try:
                import pandas as pd
                data = pd.read_csv(f, sep=" ", header=None, dtype=np.float64, engine="c",
                                   float_precision="round_trip").to_numpy()
            except ImportError:
                data = np.loadtxt(f, dtype=np.float64, ndmin=2)
    rows = data[:, 0].astype(np.int64) - 1
    cols = data[:, 1].astype(np.int64) - 1
    vals = data[:, 2]
    try:
        import pandas as pd
        diag = pd.read_csv(prefix + "sol_diag.txt", header=None, dtype=np.float64, engine="c",
                           float_precision="round_trip")[0].to_numpy()
    except ImportError:
        diag = np.loadtxt(prefix + "sol_diag.txt", dtype=np.float64, ndmin=1)
    return rows, cols, vals, diag


def run_reference(mtx_path, threads=1, physics=False, pinned_seed=None, want_factor=True,
                  timeout=600):
    """Run the reference CPU factor (cpu_implementation/driver_local.cpp main,
    :1325-1350): `driver <mtx> <threads> <out_prefix> [1]`.  Returns the
    parsed factor time and, if requested, the written factor."""
    binary = REF_BIN_PINNED if pinned_seed is not None else REF_BIN
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    env.setdefault("OMP_PROC_BIND", "close")
    if pinned_seed is not None:
        env["RCHOL_REF_SEED"] = str(pinned_seed)
    with tempfile.TemporaryDirectory() as td:
        prefix = (td + "/") if want_factor else ""
        args = [binary, mtx_path, str(threads), prefix] + (["1"] if physics else [])
        p = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference factor failed ({p.returncode}): {p.stderr[-2000:]}")
        m = re.search(r"Factorization execution time: ([0-9.eE+-]+) seconds", p.stdout)
        t = float(m.group(1)) if m else float("nan")
        m2 = re.search(r"factor nnz: (\d+)", p.stdout)
        out = dict(factor_time=t, factor_nnz=int(m2.group(1)) if m2 else -1, stdout=p.stdout)
        if want_factor:
            nm = re.search(r"number of nodes: (\d+)", p.stdout)
            n = int(nm.group(1))
            rows, cols, vals, diag = read_factor_files(prefix, n)
            out.update(rows=rows, cols=cols, vals=vals, diag=diag, n=n)
        return out
