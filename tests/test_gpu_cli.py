"""The command-line drivers keep the reference's argv forms and outputs."""
import os
import re
import subprocess

import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import GOLDEN

pytestmark = pytest.mark.gpu


def _run(args, timeout=300):
    p = subprocess.run(args, capture_output=True, text=True, timeout=timeout)
    assert p.returncode == 0, p.stdout + p.stderr
    return p.stdout


def test_driver_graph():
    out = _run([R.driver_binary("driver"), os.path.join(GOLDEN, "grid16_logw.mtx"), "512", "1", "1e-7"])
    assert "Kernel execution time:" in out and "pcg time:" in out
    it = int(re.search(r"final iteration: (\d+)", out).group(1))
    res = float(re.search(r"residual: ([0-9.e+-]+)", out).group(1))
    assert 0 < it <= 300 and res <= 1e-7


def test_driver_physics_trims_ground():
    out = _run([R.driver_binary("driver_physics"), os.path.join(GOLDEN, "cube8_sddm.mtx"), "512", "1", "7e-7"])
    m = re.search(r"normalized diff norm: ([0-9.e+-]+)", out)
    assert m and float(m.group(1)) < 1e-4


def test_driver_local_writes_reference_format(tmp_path):
    prefix = str(tmp_path) + "/"
    out = _run([R.driver_binary("driver_local"), os.path.join(GOLDEN, "cube8_sddm.mtx"), "32", prefix, "1"])
    assert "relative residual" in out
    n = 513
    rows, cols, vals, diag = O.read_factor_files(prefix, n - 1)
    assert len(diag) == n - 1
    assert np.all(rows >= cols) and np.all(vals[rows == cols] == 1.0)
    # the factor on file solves the trimmed SDDM with the oracle's PCG
    r, c, v = O_read(os.path.join(GOLDEN, "cube8_sddm.mtx"))
    colptr, rowind, val = O.triplets_to_csc(n, r, c, v)
    acp, arow, aval = O.trim_last(n, colptr, rowind, val)
    m = rows != cols
    order = np.lexsort((rows[m], cols[m]))
    lr, lc, lv = rows[m][order], cols[m][order], vals[m][order]
    lcp = np.concatenate([[0], np.cumsum(np.bincount(lc, minlength=n - 1))]).astype(np.int64)
    b = O.zero_sum_vector(n - 1, 0)
    x, info = O.pcg(n - 1, acp, arow, aval, lcp, lr.astype(np.int32), lv, diag, b, tol=1e-8)
    assert info["converged"]


def O_read(path):
    with open(path) as fh:
        fh.readline()
        n, _, nnz = map(int, fh.readline().split())
        d = np.loadtxt(fh, ndmin=2)
    return d[:, 0].astype(np.int32) - 1, d[:, 1].astype(np.int32) - 1, d[:, 2]


def test_factorization_driver_entry_point():
    L = R.lib()
    st = L.rchol_factorization_driver(os.path.join(GOLDEN, "grid12_unit.mtx").encode(), 128, 1, 1e-7, 0)
    assert st == 0


def test_driver_physics_converts_sddm_and_reads_binary_cache(tmp_path):
    """--sddm=nnz: a natural-order SDDM file is converted and ordered on the
    device (the reference's offline write_graph.jl step); a .rchb binary
    cache of the same matrix runs as the converted file does."""
    nN, r, c, v, g = R.generate("grid3d", [12, 11, 10], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                                excess_lo=0.0, excess_hi=1e-2, ordering=2, seed=2)
    m = (r < nN - 1) & (c < nN - 1)  # the SDDM without its ground vertex
    path = str(tmp_path / "sddm.mtx")
    R.write_mtx(path, nN - 1, r[m], c[m], v[m])
    out = _run([R.driver_binary("driver"), path, "512", "1", "1e-7", "--sddm=nnz", "--order_seed=2"])
    assert "converted on the device: with ground vertex" in out
    res = float(re.search(r"residual: ([0-9.e+-]+)", out).group(1))
    assert res <= 1e-7
    n0, r0, c0, v0, g0 = R.generate("grid3d", [12, 11, 10], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                                    excess_lo=0.0, excess_hi=1e-2, seed=2)
    cp, ri, val = R.csc_from_triplets(n0, r0, c0, v0)
    bpath = str(tmp_path / "c.rchb")
    R.write_bin(bpath, n0, cp, ri, val, trim_ground=True)
    out2 = _run([R.driver_binary("driver"), bpath, "512", "1", "1e-7"])
    assert float(re.search(r"residual: ([0-9.e+-]+)", out2).group(1)) <= 1e-7
    assert re.search(r"number of nodes: (\d+)", out2).group(1) == str(n0)
