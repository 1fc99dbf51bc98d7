"""Batched independent systems (many uneven Laplacians in one factor launch
and one set of PCG launches per iteration) against solving each system on
its own, and the block-diagonal factor against the oracle (bit-exact)."""
import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import OracleProblem, grid_laplacian

pytestmark = pytest.mark.gpu

SPECS = [((20, 30), 1), ((8, 8, 8), 2), ((50, 40), 3), ((6, 7, 9), 4), ((33, 5), 5)]


def _systems():
    out = []
    for dims, seed in SPECS:
        n, r, c, v, g = grid_laplacian(dims, seed=seed, wlo=1e-2, whi=1e2)
        cp, ri, val = R.csc_from_triplets(n, r, c, v)
        out.append((n, cp, ri, val, (r, c, v)))
    return out


def _zero_sum_block(offsets, k, seed):
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((offsets[-1], k))
    for s in range(len(offsets) - 1):
        B[offsets[s]:offsets[s + 1]] -= B[offsets[s]:offsets[s + 1]].mean(axis=0)
    return B


def _csc_dense(n, cp, ri, v):
    A = np.zeros((n, n))
    cols = np.repeat(np.arange(n), np.diff(cp))
    np.add.at(A, (ri, cols), v)
    return A


def _block_factor(cp, ri, val, d, lo, hi):
    """Columns lo..hi-1 of a block-diagonal factor, re-based to 0."""
    s, e = cp[lo], cp[hi]
    return dict(colptr=(cp[lo:hi + 1] - s).astype(np.int64), rowind=(ri[s:e] - lo).astype(np.int32),
                val=val[s:e].copy(), diag=d[lo:hi].copy())


@pytest.mark.parametrize("k", [1, 8])
def test_batch_matches_oracle_per_system(k):
    """Every system of the batch converges on its own scalars: per system and
    column the iteration count matches the oracle PCG run with that system's
    block of the batch factor (+-1), and so does the solution."""
    sysl = _systems()
    ctx = R.Context(seed=3, tol=1e-8)
    try:
        off = ctx.batch_set([(n, cp, ri, v) for n, cp, ri, v, _ in sysl])
        f = ctx.factor()
        fcp, fri, fval, fd = f.to_host()
        B = _zero_sum_block(off, k, 11)
        X, per, tot = ctx.batch_solve(f, B if k > 1 else B[:, 0])
        X = X.reshape(off[-1], -1)
        assert tot["status"] == 0 and tot["converged"]
        for s, (n, cp, ri, v, trip) in enumerate(sysl):
            blk = _block_factor(fcp, fri, fval, fd, off[s], off[s + 1])
            assert per[s]["relres_true"] <= 1e-8
            its = []
            for j in range(k):
                b = B[off[s]:off[s + 1], j]
                xo, io = O.pcg(n, cp, ri, v, blk["colptr"], blk["rowind"], blk["val"], blk["diag"], b,
                               tol=1e-8, max_iter=1000)
                assert io["converged"]
                its.append(io["iterations"])
                xs = X[off[s]:off[s + 1], j]
                # a Laplacian's solutions agree up to a constant shift
                dx = (xs - xs.mean()) - (xo - xo.mean())
                assert np.abs(dx).max() <= 1e-6 * np.abs(xo - xo.mean()).max()
            assert abs(per[s]["iterations"] - max(its)) <= 1
        f.free()
    finally:
        ctx.close()


def test_batch_matches_individual_solution():
    """The batch solution of each system solves that system as well as an
    independent single-system solve does."""
    sysl = _systems()
    ctx = R.Context(seed=3, tol=1e-8)
    try:
        off = ctx.batch_set([(n, cp, ri, v) for n, cp, ri, v, _ in sysl])
        f = ctx.factor()
        B = _zero_sum_block(off, 2, 12)
        X, per, tot = ctx.batch_solve(f, B)
        assert tot["converged"]
        for s, (n, cp, ri, v, trip) in enumerate(sysl):
            single = R.Context(seed=3, tol=1e-8)
            single.set_csc(n, cp, ri, v)
            fs = single.factor()
            Bs = B[off[s]:off[s + 1]]
            Xs, info = single.pcg_solve(fs, Bs)
            Xs = Xs.reshape(n, -1)
            Xb = X[off[s]:off[s + 1]]
            A = _csc_dense(n, cp, ri, v)
            res = np.linalg.norm(Bs - A @ Xb, axis=0) / np.linalg.norm(Bs, axis=0)
            assert res.max() <= 1.01e-8
            # different factors (other Philox vertex keys) and both stopped at
            # relres 1e-8: the solutions agree to well inside cond(A) * 1e-8
            scale = np.abs(Xs - Xs.mean(axis=0)).max()
            np.testing.assert_allclose(Xb - Xb.mean(axis=0), Xs - Xs.mean(axis=0), rtol=0, atol=1e-4 * scale)
            fs.free()
            single.close()
        f.free()
    finally:
        ctx.close()


def test_batch_factor_is_block_diagonal_and_bitexact():
    sysl = _systems()
    ctx = R.Context(seed=9)
    try:
        off = ctx.batch_set([(n, cp, ri, v) for n, cp, ri, v, _ in sysl])
        f = ctx.factor()
        cp, ri, val, d = f.to_host()
        nt, colptr, rowind, v = ctx.matrix()
        P = OracleProblem.__new__(OracleProblem)
        P.n = nt
        P.trim = False
        P.colptr, P.rowind, P.val = colptr, rowind, v
        P.lcp, P.lrow, P.lval = O.lower_triangle(nt, colptr, rowind, v)
        P.dep = O.dependency_counts(nt, colptr, rowind)
        orc = O.factor(nt, P.lcp, P.lrow, P.lval, P.dep, seed=9)
        assert np.array_equal(ri, orc["rowind"]) and np.array_equal(val, orc["val"])
        assert np.array_equal(d, orc["diag"])
        # no entry couples two systems
        cols = np.repeat(np.arange(nt), np.diff(cp))
        sys_of = np.searchsorted(off, np.arange(nt), side="right") - 1
        assert np.array_equal(sys_of[cols], sys_of[ri])
        f.free()
    finally:
        ctx.close()


def test_batch_rejects_tiny_systems():
    ctx = R.Context()
    try:
        n, r, c, v, _ = grid_laplacian((4, 4), seed=1)
        cp, ri, val = R.csc_from_triplets(n, r, c, v)
        with pytest.raises(R.RcholError):
            ctx.batch_set([(n, cp, ri, val)])
    finally:
        ctx.close()
