"""Shared test helpers: inputs, oracle runs, comparisons."""
import os

import numpy as np

import pyoracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def grid_laplacian(dims, seed=0, log_weights=True, wlo=1e-2, whi=1e2, excess_frac=0.0, excess_hi=1e-1):
    """numpy-built grid Laplacian in ascending-nnz order (seeded tie-break),
    with a ground vertex appended when excess_frac > 0.  Returns
    (n, rows, cols, vals, has_ground)."""
    rng = np.random.default_rng(seed)
    n = int(np.prod(dims))
    idx = np.arange(n).reshape(dims[::-1])
    a, b = [], []
    for ax in range(len(dims)):
        s0 = [slice(None)] * len(dims)
        s1 = [slice(None)] * len(dims)
        s0[ax] = slice(0, -1)
        s1[ax] = slice(1, None)
        a.append(idx[tuple(s0)].ravel())
        b.append(idx[tuple(s1)].ravel())
    a = np.concatenate(a)
    b = np.concatenate(b)
    w = np.exp(rng.uniform(np.log(wlo), np.log(whi), len(a))) if log_weights else np.ones(len(a))
    deg = np.bincount(a, minlength=n) + np.bincount(b, minlength=n)
    perm = rng.permutation(n)
    order = perm[np.argsort(deg[perm], kind="stable")]
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    a2, b2 = inv[a], inv[b]
    wd = np.zeros(n)
    np.add.at(wd, a2, w)
    np.add.at(wd, b2, w)
    exc = np.zeros(n)
    if excess_frac > 0:
        pick = rng.random(n) < excess_frac
        exc[pick] = rng.uniform(0, excess_hi, pick.sum()) * wd[pick]
    rows = [a2, b2, np.arange(n)]
    cols = [b2, a2, np.arange(n)]
    vals = [-w, -w, wd + exc]
    N = n
    if (exc > 0).any():
        g = np.nonzero(exc > 0)[0]
        rows += [g, np.full(len(g), n), np.array([n])]
        cols += [np.full(len(g), n), g, np.array([n])]
        vals += [-exc[g], -exc[g], np.array([exc.sum()])]
        N = n + 1
    return (N, np.concatenate(rows).astype(np.int32), np.concatenate(cols).astype(np.int32),
            np.concatenate(vals), N != n)


class OracleProblem:
    """The oracle's preprocessing of a triplet matrix (pre_process.hpp)."""

    def __init__(self, n, rows, cols, vals, trim=False):
        self.n = n
        self.trim = trim
        self.colptr, self.rowind, self.val = O.triplets_to_csc(n, rows, cols, vals)
        self.lcp, self.lrow, self.lval = O.lower_triangle(n, self.colptr, self.rowind, self.val)
        self.dep = O.dependency_counts(n, self.colptr, self.rowind)
        if trim:
            self.acp, self.arow, self.aval = O.trim_last(n, self.colptr, self.rowind, self.val)
            self.ns = n - 1
        else:
            self.acp, self.arow, self.aval = self.colptr, self.rowind, self.val
            self.ns = n

    def factor(self, seed=1, mode=O.MODE_B200):
        f = O.factor(self.n, self.lcp, self.lrow, self.lval, self.dep, mode=mode, seed=seed)
        return trim_factor(f, self.n) if self.trim else f

    def pcg(self, f, b, tol=1e-6, max_iter=1000, stop_rule=O.STOP_RELRES, nthreads=1):
        return O.pcg(self.ns, self.acp, self.arow, self.aval, f["colptr"], f["rowind"], f["val"], f["diag"], b,
                     tol=tol, max_iter=max_iter, stop_rule=stop_rule, nthreads=nthreads)


def trim_factor(f, n):
    """Drop the last vertex (ground) from an oracle factor."""
    cp, ri, v = f["colptr"], f["rowind"], f["val"]
    cols = np.repeat(np.arange(n), np.diff(cp))
    keep = (ri < n - 1) & (cols < n - 1)
    out = dict(f)
    out["colptr"] = np.concatenate([[0], np.cumsum(np.bincount(cols[keep], minlength=n - 1))]).astype(np.int64)
    out["rowind"] = ri[keep].astype(np.int32)
    out["val"] = v[keep].copy()
    out["diag"] = f["diag"][:n - 1].copy()
    return out


def read_reference_factor(prefix, n):
    """Strict CSC (per column, rows ascending) + D from the reference's
    l_sol.mtx / sol_diag.txt."""
    rows, cols, vals, diag = O.read_factor_files(prefix, n)
    m = rows != cols
    assert np.all(vals[~m] == 1.0), "unit diagonal"
    assert np.all(rows >= cols), "row >= col"
    r, c, v = rows[m], cols[m], vals[m]
    order = np.lexsort((r, c))
    r, c, v = r[order], c[order], v[order]
    cp = np.zeros(n + 1, np.int64)
    np.add.at(cp, c + 1, 1)
    cp = np.cumsum(cp)
    return cp, r.astype(np.int32), v, diag


def zero_sum_normal(n, seed):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(n)
    return b - b.mean()


def disconnected_laplacian():
    """A 12^2 grid, a 6^3 grid and one vertex with no edges (an explicit zero
    diagonal), in one ascending-degree order with a seeded tie-break.
    Returns (n, rows, cols, vals, iso, comp1, comp2): the isolated vertex's
    index and each grid's vertex indices in the combined order."""
    n1, r1, c1, v1, _ = grid_laplacian((12, 12), seed=41)
    n2, r2, c2, v2, _ = grid_laplacian((6, 6, 6), seed=42)
    n = n1 + n2 + 1
    rows = np.concatenate([r1, r2 + n1, [n - 1]]).astype(np.int64)
    cols = np.concatenate([c1, c2 + n1, [n - 1]]).astype(np.int64)
    vals = np.concatenate([v1, v2, [0.0]])
    deg = np.bincount(rows[rows != cols], minlength=n)
    rng = np.random.default_rng(43)
    perm = rng.permutation(n)
    order = perm[np.argsort(deg[perm], kind="stable")]
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    r, c = inv[rows].astype(np.int32), inv[cols].astype(np.int32)
    return n, r, c, vals, int(inv[n - 1]), inv[:n1], inv[n1:n1 + n2]


def per_component_rhs(n, comp1, comp2):
    """Zero sum on each grid component, zero on the isolated vertex."""
    b = np.zeros(n)
    b[comp1] = zero_sum_normal(len(comp1), 44)
    b[comp2] = zero_sum_normal(len(comp2), 45)
    return b
