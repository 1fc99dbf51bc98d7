"""Statistical parity with the reference CPU factor (parallel mode).

The reference seeds each thread from std::random_device, so its factor
varies run to run.  Over 5 runs of the compiled reference
(oracle/_ref/rchol_ref_cpu, all host threads) and 5 GPU seeds on the same
ordered input: the GPU factor nnz lies within +-5% of the reference median,
and PCG iterations (oracle PCG on the reference factors, GPU PCG on the GPU
factors, same right-hand side, true relative residual 1e-6) within +-10% of
the reference median (medians compared; single runs within +-25% of the
reference's range).  Every solve reaches the tolerance.
"""
import os
import tempfile

import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import OracleProblem, read_reference_factor

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(O.REF_BIN), reason="reference CPU factor not built (oracle/_ref)")
@pytest.mark.parametrize("config", ["grid2d_256_unit", "grid3d_32_sddm", "chunglu_200k", "grid27_48_sddm",
                                    pytest.param("grid3d_128_sddm", marks=pytest.mark.slow)])
def test_statistical_parity_with_reference(config):
    """grid3d_128_sddm is the benchmark's headline input itself (128^3 SDDM,
    2,097,152 unknowns); it takes a few minutes of host time.  chunglu_200k
    and grid27_48_sddm are the power-law and anisotropic 27-point families
    of the secondary benchmarks at a size the host finishes in seconds."""
    if config == "grid2d_256_unit":
        n, r, c, v, g = R.generate("grid2d", [256, 256], seed=0)
    elif config == "chunglu_200k":
        n, r, c, v, g = R.generate("chunglu", [200_000, 2_000_000, 2, 20_000], wlo=1.0, whi=10.0, seed=3)
    elif config == "grid27_48_sddm":
        n, r, c, v, g = R.generate("grid3d27", [48, 48, 48], wlo=0.1, whi=10.0, log_weights=True, aniso_z=100.0,
                                   excess_frac=1.0, excess_lo=1e-4, excess_hi=1e-4, seed=5)
    else:
        side = 128 if config == "grid3d_128_sddm" else 32
        n, r, c, v, g = R.generate("grid3d", [side] * 3, wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                                   excess_lo=0.0, excess_hi=1e-2, seed=2)
    P = OracleProblem(n, r, c, v, trim=g)
    threads = str(max(1, min(os.cpu_count() or 1, 16)))
    ref_nnz, ref_its = [], []
    b = O.zero_sum_vector(P.ns, 0)
    with tempfile.TemporaryDirectory() as td:
        mtx = os.path.join(td, "a.mtx")
        R.write_mtx(mtx, n, r, c, v)
        for run in range(5):
            out = O.run_reference(mtx, threads=int(threads), physics=g, want_factor=True)
            cp, ri, val, d = read_reference_factor_from(out, n)
            f = dict(colptr=cp, rowind=ri, val=val, diag=d)
            if g:
                from helpers import trim_factor
                f = trim_factor(f, n)
            ref_nnz.append(len(f["rowind"]))
            _, info = P.pcg(f, b, tol=1e-6, nthreads=int(threads))
            assert info["converged"]
            ref_its.append(info["iterations"])
    gpu_nnz, gpu_its = [], []
    ctx = R.Context()
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        for seed in range(1, 6):
            ctx.set_opts(seed=seed, tol=1e-6)
            f = ctx.factor()
            gpu_nnz.append(f.info().nnz_strict)
            x, info = ctx.pcg_solve(f, b)
            assert info["converged"] and info["relres_true"] <= 1e-6
            gpu_its.append(info["iterations"])
            f.free()
    finally:
        ctx.close()
    mn, mi = np.median(ref_nnz), np.median(ref_its)
    # every GPU factor's nnz within +-5% of the reference median; the GPU's
    # median iteration count within +-10% of the reference median (single
    # runs scatter by more than that on both sides: the reference itself
    # spans 34..39 iterations on the 256^2 grid)
    assert np.all(np.abs(np.array(gpu_nnz) - mn) <= 0.05 * mn), (gpu_nnz, ref_nnz)
    assert abs(np.median(gpu_its) - mi) <= max(0.10 * mi, 1.0), (gpu_its, ref_its)
    assert max(gpu_its) <= 1.25 * max(ref_its) and min(gpu_its) >= 0.75 * min(ref_its), (gpu_its, ref_its)


def read_reference_factor_from(out, n):
    rows, cols, vals, diag = out["rows"], out["cols"], out["vals"], out["diag"]
    m = rows != cols
    order = np.lexsort((rows[m], cols[m]))
    r, c, v = rows[m][order], cols[m][order], vals[m][order]
    cp = np.concatenate([[0], np.cumsum(np.bincount(c, minlength=n))]).astype(np.int64)
    return cp, r.astype(np.int32), v, diag
