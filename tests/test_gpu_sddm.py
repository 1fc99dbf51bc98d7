"""SDDM -> ordered Laplacian on the device (rchol_set_sddm) against the
oracle's restatement of the reference's physics preprocessing
(cpu_implementation/write_graph.jl:98-183): the matrix, the permutation and
the ground vertex bit for bit; then a solve in the input's numbering."""
import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R

pytestmark = pytest.mark.gpu


def _natural_sddm(kind, dims, **kw):
    nN, r, c, v, g = R.generate(kind, dims, ordering=2, **kw)
    if g:
        m = (r < nN - 1) & (c < nN - 1)
        return nN - 1, r[m], c[m], v[m]
    return nN, r, c, v


@pytest.mark.parametrize("case,ordering", [
    ("cube_sddm", R.ORDER_NNZ_SORT), ("cube27_sddm", R.ORDER_RANDOM), ("grid_laplacian", R.ORDER_NNZ_SORT),
    ("cube_sddm", R.ORDER_GIVEN),
])
def test_set_sddm_matches_oracle(case, ordering):
    if case == "cube_sddm":
        n, r, c, v = _natural_sddm("grid3d", [11, 10, 9], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                                   excess_lo=0.0, excess_hi=1e-2, seed=2)
    elif case == "cube27_sddm":
        n, r, c, v = _natural_sddm("grid3d27", [7, 6, 8], wlo=0.1, whi=10.0, log_weights=True, aniso_z=100.0,
                                   excess_frac=1.0, excess_lo=1e-4, excess_hi=1e-4, seed=5)
    else:
        n, r, c, v = _natural_sddm("grid2d", [23, 19], wlo=1e-2, whi=1e2, log_weights=True, seed=3)
    seed = 17
    N, cp, ri, val, perm, g = O.sddm_to_laplacian(n, r, c, v, ordering, seed)
    ctx = R.Context()
    try:
        dperm, dg = ctx.set_sddm(n, r, c, v, ordering=ordering, order_seed=seed)
        Nd, cpd, rid, vald = ctx.matrix()
        assert dg == g and Nd == N
        assert np.array_equal(dperm, perm)
        assert np.array_equal(cpd, cp) and np.array_equal(rid, ri) and np.array_equal(vald, val)
    finally:
        ctx.close()


def test_set_sddm_appends_missing_diagonal_and_rejects_non_dominant():
    n, r, c, v = _natural_sddm("grid2d", [12, 9], seed=4)
    off = r != c
    r, c, v = r[off], c[off], np.abs(v[off])  # adjacency only: the diagonal is appended
    N, cp, ri, val, perm, g = O.sddm_to_laplacian(n, r, c, v, 1, 3)
    ctx = R.Context()
    try:
        dperm, dg = ctx.set_sddm(n, r, c, v, ordering=R.ORDER_NNZ_SORT, order_seed=3)
        Nd, cpd, rid, vald = ctx.matrix()
        assert not dg and not g and Nd == N == n
        assert np.array_equal(cpd, cp) and np.array_equal(rid, ri) and np.array_equal(vald, val)
        # a diagonal below the off-diagonal sum: not diagonally dominant
        rr = np.concatenate([r, np.arange(n)])
        cc = np.concatenate([c, np.arange(n)])
        vv = np.concatenate([-v, np.full(n, 0.5)])
        with pytest.raises(R.RcholError) as e:
            ctx.set_sddm(n, rr, cc, vv)
        assert e.value.status == 8
    finally:
        ctx.close()


def test_set_sddm_solve_in_input_numbering():
    """Factor and solve the converted system; mapping the right-hand side
    through the permutation gives the SDDM's own solution."""
    n, r, c, v = _natural_sddm("grid3d", [16, 15, 14], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                               excess_lo=0.0, excess_hi=1e-2, seed=2)
    ctx = R.Context(seed=5, tol=1e-8)
    try:
        perm, g = ctx.set_sddm(n, r, c, v, ordering=R.ORDER_NNZ_SORT, order_seed=2)
        assert g
        f = ctx.factor()
        b = np.random.default_rng(9).standard_normal(n)
        bp = np.empty(n)
        bp[perm] = b
        xp, info = ctx.pcg_solve(f, bp)
        assert info["converged"] and info["relres_true"] <= 1e-8
        x = xp[perm]
        Ax = np.zeros(n)
        np.add.at(Ax, r, v * x[c])
        assert np.linalg.norm(b - Ax) / np.linalg.norm(b) <= 1.01e-8
        f.free()
    finally:
        ctx.close()


@pytest.mark.parametrize("ordering", [R.ORDER_RCM, R.ORDER_ND])
def test_set_sddm_host_orderings(ordering):
    """RCM and nested dissection are computed on the host from the pattern
    (rchol_ordering) and applied by the device conversion; the factor of the
    reordered system solves the input's system."""
    n, r, c, v = _natural_sddm("grid3d", [13, 12, 11], wlo=1e-3, whi=1e3, log_weights=True, excess_frac=0.05,
                               excess_lo=0.0, excess_hi=1e-2, seed=2)
    order = R.ordering(ordering, n, r, c)
    N, cp, ri, val, perm, g = O.sddm_to_laplacian(n, r, c, v, order=order)
    ctx = R.Context(seed=6, tol=1e-8)
    try:
        dperm, dg = ctx.set_sddm(n, r, c, v, ordering=ordering)
        Nd, cpd, rid, vald = ctx.matrix()
        assert dg == g and np.array_equal(dperm, perm)
        assert np.array_equal(cpd, cp) and np.array_equal(rid, ri) and np.array_equal(vald, val)
        f = ctx.factor()
        b = np.random.default_rng(1).standard_normal(n)
        bp = np.empty(n)
        bp[dperm] = b
        xp, info = ctx.pcg_solve(f, bp)
        assert info["converged"]
        f.free()
    finally:
        ctx.close()
