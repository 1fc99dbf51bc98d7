"""Host logic of the product library, no GPU needed: preprocessing (a1),
MatrixMarket IO, generators and ground conversion (a2), the C-ABI surface."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import grid_laplacian

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rchol.h")


def test_library_exports_every_declared_symbol():
    text = open(HEADER).read()
    declared = sorted(set(re.findall(r"\b(rchol_[a-z0-9_]+)\s*\(", text)))
    assert declared, "no declarations parsed"
    L = ctypes.CDLL(R.LIB_PATH)
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(R.EXPORTS) == declared


def test_nm_shows_c_linkage():
    out = subprocess.run(["nm", "-D", "--defined-only", R.LIB_PATH], capture_output=True, text=True).stdout
    for s in R.EXPORTS:
        assert re.search(rf"\bT {s}$", out, re.M), s


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(R.RcholError) as e:
        R.Context()
    assert e.value.status == 7  # RCHOL_ERR_NO_DEVICE: no CPU fallback


def test_option_defaults_and_validation():
    """rchol_create checks the options before it looks for a device: bad
    values are RCHOL_ERR_INVALID (1) on any machine, good ones get as far as
    the device check (RCHOL_ERR_NO_DEVICE, 7, without a GPU)."""
    import torch
    o = R.default_opts()
    assert o.sched_epl == 0  # automatic schedule width
    assert o.spmv_layout == R.SPMV_AUTO
    lib = R.lib()
    good = 0 if torch.cuda.is_available() else 7

    def create(**kw):
        h = ctypes.c_void_p()
        st = lib.rchol_create(ctypes.byref(h), ctypes.byref(R.default_opts(**kw)))
        if st == 0:
            lib.rchol_destroy(h)
        return st

    for kw in (dict(sched_epl=0), dict(sched_epl=3), dict(sched_epl=64), dict(spmv_layout=R.SPMV_CSR)):
        assert create(**kw) == good, kw
    for kw in (dict(sched_epl=-1), dict(sched_epl=65), dict(spmv_layout=2), dict(spmv_layout=-1)):
        assert create(**kw) == 1, kw


@pytest.mark.parametrize("case", ["grid2d", "grid3d_sddm", "with_duplicates", "no_diagonal", "positive_offdiag"])
def test_preprocessing_matches_oracle(case):
    rng = np.random.default_rng(1)
    if case == "grid2d":
        n, r, c, v, _ = grid_laplacian((17, 13), seed=2)
    elif case == "grid3d_sddm":
        n, r, c, v, _ = grid_laplacian((6, 5, 4), seed=3, excess_frac=0.2)
    elif case == "with_duplicates":
        n, r, c, v, _ = grid_laplacian((9, 9), seed=4)
        k = rng.choice(len(r), 40, replace=False)
        r, c, v = np.concatenate([r, r[k]]), np.concatenate([c, c[k]]), np.concatenate([v, v[k] * 0.5])
    elif case == "no_diagonal":
        # graph adjacency only: the diagonal is appended as sum |off| (pre_process.hpp:222-241)
        n, r, c, v, _ = grid_laplacian((8, 11), seed=5)
        m = r != c
        r, c, v = r[m], c[m], np.abs(v[m])
    else:
        n, r, c, v, _ = grid_laplacian((7, 7), seed=6)
        v = np.where(r != c, np.abs(v), v)  # signs are normalised to -|v|
    perm = rng.permutation(len(r))
    r, c, v = r[perm], c[perm], v[perm]
    got = R.csc_from_triplets(n, r, c, v)
    exp = O.triplets_to_csc(n, r, c, v)
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)


def test_preprocessing_rejects_nonfinite():
    n, r, c, v, _ = grid_laplacian((4, 4), seed=1)
    v = v.copy()
    v[3] = np.nan
    with pytest.raises(R.RcholError) as e:
        R.csc_from_triplets(n, r, c, v)
    assert e.value.status == 8


def test_mtx_roundtrip_and_symmetric_generalisation():
    n, r, c, v, _ = grid_laplacian((6, 7), seed=7)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "a.mtx")
        R.write_mtx(p, n, r, c, v)
        n2, r2, c2, v2 = R.read_mtx(p)
        assert n2 == n and np.array_equal(r2, r) and np.array_equal(c2, c) and np.array_equal(v2, v)
        # a symmetric file holding only the lower triangle expands to both
        low = r >= c
        q = os.path.join(td, "s.mtx")
        with open(q, "w") as f:
            f.write("%%MatrixMarket matrix coordinate real symmetric\n% comment\n")
            f.write(f"{n} {n} {int(low.sum())}\n")
            for a, b, x in zip(r[low], c[low], v[low]):
                f.write(f"{a + 1} {b + 1} {x:.17g}\n")
        n3, r3, c3, v3 = R.read_mtx(q)
        A = np.zeros((n, n))
        np.add.at(A, (r, c), v)
        B = np.zeros((n, n))
        np.add.at(B, (r3, c3), v3)
        assert np.array_equal(A, B)


def test_generator_grid2d_config1_shape():
    n, r, c, v, g = R.generate("grid2d", [256, 256], seed=0)
    assert n == 65536 and len(r) == 326656 and not g
    colptr, rowind, val = R.csc_from_triplets(n, r, c, v)
    sums = np.add.reduceat(val, colptr[:-1])
    assert np.abs(sums).max() < 1e-12
    deg = np.diff(colptr)
    assert np.all(np.diff(deg) >= 0)  # ascending nnz ordering


def test_generator_sddm_ground_vertex():
    n, r, c, v, g = R.generate("grid3d", [10, 10, 10], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                               excess_lo=0.0, excess_hi=1e-2, seed=2)
    assert g and n == 1001
    colptr, rowind, val = R.csc_from_triplets(n, r, c, v)
    # Laplacian with the ground: every column sums to ~0
    sums = np.add.reduceat(val, colptr[:-1])
    scale = np.add.reduceat(np.abs(val), colptr[:-1])
    assert np.all(np.abs(sums) <= 1e-12 * scale)
    # the ground vertex is last and connects only to rows with excess
    last = rowind[colptr[n - 1]:colptr[n]]
    assert last[-1] == n - 1 and 0 < len(last) - 1 < 0.15 * (n - 1)
    # the SDDM part (ground trimmed) is ordered by ascending nnz
    ocp, orow, _ = O.trim_last(n, colptr, rowind, val)
    deg = np.diff(ocp)
    assert np.all(np.diff(deg) >= 0)


def test_generator_27pt_and_chunglu():
    n, r, c, v, g = R.generate("grid3d27", [6, 6, 6], wlo=0.1, whi=10, log_weights=True, aniso_z=100.0,
                               excess_frac=1.0, excess_lo=1e-4, excess_hi=1e-4, seed=5)
    assert g and n == 217
    colptr, _, _ = R.csc_from_triplets(n, r, c, v)
    assert colptr[-1] == 2 * (13 * 4 * 4 * 4 + 0) + 0 or colptr[-1] > 0
    n2, r2, c2, v2, g2 = R.generate("chunglu", [2000, 8000, 2, 200], wlo=1, whi=10, seed=3)
    assert not g2 and 1000 < n2 <= 2000
    colptr2, rowind2, val2 = R.csc_from_triplets(n2, r2, c2, v2)
    assert np.abs(np.add.reduceat(val2, colptr2[:-1])).max() < 1e-9


def test_generator_deterministic():
    a = R.generate("grid3d", [5, 6, 7], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.1, excess_hi=1e-2,
                   seed=11)
    b = R.generate("grid3d", [5, 6, 7], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.1, excess_hi=1e-2,
                   seed=11)
    for x, y in zip(a[1:4], b[1:4]):
        assert np.array_equal(x, y)


def test_cli_usage_errors_without_gpu():
    for name in ["driver", "driver_physics", "driver_local"]:
        p = subprocess.run([R.driver_binary(name)], capture_output=True, text=True)
        assert p.returncode == 1 and "argument count not correct" in p.stdout


@pytest.mark.parametrize("kind,dims,kw", [
    ("grid3d", [14, 13, 12], dict(wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05, excess_lo=0.0,
                                  excess_hi=1e-2, seed=2)),
    ("grid2d", [33, 17], dict(seed=0)),
    ("grid3d27", [9, 8, 7], dict(wlo=0.1, whi=10.0, log_weights=True, aniso_z=100.0, excess_frac=1.0,
                                 excess_lo=1e-4, excess_hi=1e-4, seed=5)),
])
def test_oracle_input_generator_matches_library(kind, dims, kw):
    """The CPU legs of bench.py build their input with oracle/gen_inputs.c
    (never loading the product library); it must give the library
    generator's triplets bit for bit."""
    a = R.generate(kind, dims, **kw)
    b = O.generate_grid(kind, dims, **kw)
    assert a[0] == b[0] and a[4] == b[4]
    for x, y in zip(a[1:4], b[1:4]):
        assert np.array_equal(x, y)


def test_bench_arms_share_the_input():
    """Both bench arms print the same config, including the input checksum."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    B = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(B)
    cfg = dict(B.CONFIGS["c2"], dims=[12, 12, 12])
    Wp = B.build_workload(cfg, product=True)
    Wo = B.build_workload(cfg, product=False)
    assert B.workload_config(cfg, Wp) == B.workload_config(cfg, Wo)


@pytest.mark.parametrize("kind,dims,kw", [
    ("grid3d", [9, 8, 7], dict(wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05, excess_lo=0.0, excess_hi=1e-2,
                               seed=2)),
    ("grid3d27", [6, 7, 5], dict(wlo=0.1, whi=10.0, log_weights=True, aniso_z=100.0, excess_frac=1.0,
                                 excess_lo=1e-4, excess_hi=1e-4, seed=5)),
    ("grid2d", [15, 13], dict(seed=5)),
])
def test_sddm_conversion_oracle_matches_generator(kind, dims, kw):
    """The oracle's restatement of the physics preprocessing (write_graph.jl:
    98-183), applied to the natural-order SDDM, gives the generator's ordered
    Laplacian: same order, same pattern, ground values within rounding (the
    generator knows each excess, the conversion recovers it as a column sum)."""
    nN, rN, cN, vN, gN = R.generate(kind, dims, ordering=2, **kw)
    n0, r0, c0, v0, g0 = R.generate(kind, dims, ordering=0, **kw)
    if gN:  # strip the natural-order ground vertex: back to the SDDM
        m = (rN < nN - 1) & (cN < nN - 1)
        rN, cN, vN, n = rN[m], cN[m], vN[m], nN - 1
    else:
        n = nN
    N, cp, ri, val, perm, g = O.sddm_to_laplacian(n, rN, cN, vN, 1, kw["seed"])
    cp0, ri0, val0 = O.triplets_to_csc(n0, r0, c0, v0)
    assert N == n0 and g == g0
    assert np.array_equal(cp, cp0) and np.array_equal(ri, ri0)
    np.testing.assert_allclose(val, val0, rtol=1e-10, atol=0)


def test_parallel_mtx_reader_keeps_file_order(tmp_path):
    """The chunked parallel MatrixMarket parse returns the entries in file
    order (blank and comment lines in the body skipped), as the sequential
    reader of the test oracle does."""
    n, r, c, v, g = R.generate("grid3d", [30, 29, 28], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                               excess_lo=0.0, excess_hi=1e-2, seed=2)
    path = str(tmp_path / "a.mtx")
    O.write_mtx(path, n, r, c, v)
    n2, r2, c2, v2 = R.read_mtx(path)
    assert n2 == n and np.array_equal(r2, r) and np.array_equal(c2, c) and np.array_equal(v2, v)
    # a symmetric file with comments and a blank line is generalised
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n% comment\n3 3 4\n1 1 2.5\n\n2 1 -1\n3 2 -0.5\n"
                "3 3 4\n")
    n3, r3, c3, v3 = R.read_mtx(path)
    assert n3 == 3 and list(r3) == [0, 1, 2, 2, 0, 1] and list(c3) == [0, 0, 1, 2, 1, 2]
    assert list(v3) == [2.5, -1.0, -0.5, 4.0, -1.0, -0.5]
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n3 3 3\n1 1 1\n2 2 1\n")
    with pytest.raises(R.RcholError):
        R.read_mtx(path)


def test_binary_matrix_cache_roundtrip(tmp_path):
    n, r, c, v, g = R.generate("grid2d", [40, 33], wlo=1e-2, whi=1e2, log_weights=True, seed=8)
    cp, ri, val = R.csc_from_triplets(n, r, c, v)
    path = str(tmp_path / "a.rchb")
    R.write_bin(path, n, cp, ri, val, trim_ground=True)
    n2, cp2, ri2, val2, tr = R.read_bin(path)
    assert n2 == n and tr and np.array_equal(cp2, cp) and np.array_equal(ri2, ri) and np.array_equal(val2, val)
    with open(path, "r+b") as f:  # corrupt an index: rejected, not trusted
        f.seek(32 + 4 * (n + 1))
        f.write(np.array([n + 7], np.int32).tobytes())
    with pytest.raises(R.RcholError):
        R.read_bin(path)


def _etree_height(n, rows, cols, order):
    """Height of the elimination tree of the pattern in `order` (Liu's
    algorithm with path compression)."""
    pos = np.empty(n, np.int64)
    pos[order] = np.arange(n)
    pr, pc = pos[rows], pos[cols]
    m = pr > pc
    # rows of the permuted lower triangle, by column... the etree needs, for
    # each row i, its columns j < i
    byrow = [[] for _ in range(n)]
    for i, j in zip(pr[m], pc[m]):
        byrow[i].append(j)
    parent = [-1] * n
    anc = [-1] * n
    for i in range(n):
        for j in byrow[i]:
            while j != -1 and j < i:
                nxt = anc[j]
                anc[j] = i
                if nxt == -1:
                    parent[j] = i
                j = nxt
    height = [0] * n
    for i in range(n):
        if parent[i] != -1:
            height[parent[i]] = max(height[parent[i]], height[i] + 1)
    return max(height)


def test_host_orderings():
    """RCM narrows the bandwidth of a randomly ordered grid; nested dissection
    gives a shallow elimination tree; both are permutations, also of a
    disconnected graph."""
    n, r, c, v, g = R.generate("grid3d", [16, 15, 14], ordering=1, seed=3)
    pos = lambda o: np.argsort(o)
    m = r != c
    rcm = R.ordering(R.ORDER_RCM, n, r, c)
    nd = R.ordering(R.ORDER_ND, n, r, c)
    for o in (rcm, nd):
        assert np.array_equal(np.sort(o), np.arange(n))
    bw = lambda o: np.abs(pos(o)[r[m]] - pos(o)[c[m]]).max()
    assert bw(rcm) < 0.1 * bw(np.arange(n))
    n2, r2, c2, v2, g2 = R.generate("grid2d", [40, 40], seed=4, ordering=2)
    h_nd = _etree_height(n2, r2, c2, R.ordering(R.ORDER_ND, n2, r2, c2))
    h_rcm = _etree_height(n2, r2, c2, R.ordering(R.ORDER_RCM, n2, r2, c2))
    assert h_nd < 0.6 * h_rcm
    # two disjoint grids
    rr = np.concatenate([r2, r2 + n2])
    cc = np.concatenate([c2, c2 + n2])
    for kind in (R.ORDER_RCM, R.ORDER_ND):
        o = R.ordering(kind, 2 * n2, rr, cc)
        assert np.array_equal(np.sort(o), np.arange(2 * n2))
