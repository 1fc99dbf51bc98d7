"""PCG and its kernels (through the C-ABI) against the oracle.

Tolerances: the SpMV and the preconditioner apply in FP64 agree with the
oracle to 1e-12 relative (different summation order); with the FP32 factor
copy to 2e-5 relative.  PCG on bit-identical factors takes the same number
of iterations as the oracle's PCG within +-1 and reaches the stated true
relative residual.
"""
import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import OracleProblem, disconnected_laplacian, grid_laplacian, per_component_rhs, zero_sum_normal

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    n, r, c, v, g = grid_laplacian((16, 16, 16), seed=21, excess_frac=0.05, wlo=1e-3, whi=1e3)
    P = OracleProblem(n, r, c, v, trim=g)
    ctx = R.Context(seed=5, precision=R.PREC_FP32_FACTOR)
    ctx.set_triplets(n, r, c, v, trim_ground=g)
    f = ctx.factor()
    orc = P.factor(seed=5)
    yield P, ctx, f, orc
    f.free()
    ctx.close()


def _csr_matvec(P, x):
    y = np.zeros_like(x)
    for j in range(P.ns):
        s, e = P.acp[j], P.acp[j + 1]
        y[j] = np.dot(P.aval[s:e], x[P.arow[s:e]])
    return y


def test_factor_matches_oracle(problem):
    P, ctx, f, orc = problem
    cp, ri, val, d = f.to_host()
    assert np.array_equal(ri, orc["rowind"]) and np.array_equal(val, orc["val"]) and np.array_equal(d, orc["diag"])


def test_spmv(problem):
    P, ctx, f, orc = problem
    X = np.random.default_rng(1).standard_normal((P.ns, 4))
    Y = ctx.spmv(X)
    for k in range(4):
        ref = O.spmv(P.ns, P.acp, P.arow, P.aval, X[:, k])
        np.testing.assert_allclose(Y[:, k], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("k", [1, 2, 8, 32])
def test_precond_apply_fp64(problem, k):
    P, ctx, f, orc = problem
    R_ = np.random.default_rng(k).standard_normal((P.ns, k))
    Z = ctx.precond_apply(f, R_ if k > 1 else R_[:, 0])
    Z = Z.reshape(P.ns, -1)
    for c in range(k):
        ref = O.precond_apply(P.ns, orc["colptr"], orc["rowind"], orc["val"], orc["diag"], R_[:, c])
        np.testing.assert_allclose(Z[:, c], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_precond_apply_fp32(problem):
    P, ctx, f, orc = problem
    r = np.random.default_rng(3).standard_normal(P.ns)
    z = ctx.precond_apply(f, r, fp32=True)
    ref = O.precond_apply(P.ns, orc["colptr"], orc["rowind"], orc["val"], orc["diag"], r)
    np.testing.assert_allclose(z, ref, rtol=2e-5, atol=2e-5 * np.abs(ref).max())


@pytest.mark.parametrize("precision", [R.PREC_FP64, R.PREC_FP32_FACTOR])
def test_pcg_vs_oracle(problem, precision):
    P, ctx, f, orc = problem
    b = zero_sum_normal(P.ns, 7)
    ctx.set_opts(precision=precision, tol=1e-8, stop_rule=R.STOP_RELRES)
    x, info = ctx.pcg_solve(f, b)
    xo, io = P.pcg(orc, b, tol=1e-8)
    assert info["status"] == 0 and info["converged"]
    assert info["relres_true"] <= 1e-8
    true = np.linalg.norm(b - _csr_matvec(P, x)) / np.linalg.norm(b)
    assert true <= 1.05e-8
    assert abs(info["iterations"] - io["iterations"]) <= (1 if precision == R.PREC_FP64 else 3)
    np.testing.assert_allclose(x, xo, rtol=0, atol=1e-6 * np.abs(xo).max())


def test_pcg_reference_stop_rule(problem):
    P, ctx, f, orc = problem
    b = O.zero_sum_vector(P.ns, 0)
    ctx.set_opts(precision=R.PREC_FP64, tol=1e-7, stop_rule=R.STOP_PRECOND, max_iter=300)
    x, info = ctx.pcg_solve(f, b)
    xo, io = P.pcg(orc, b, tol=1e-7, max_iter=300, stop_rule=O.STOP_PRECOND)
    assert abs(info["iterations"] - io["iterations"]) <= 1
    assert info["precond_ratio"] <= 1e-7
    ctx.set_opts(stop_rule=R.STOP_RELRES, max_iter=1000, tol=1e-6)


@pytest.mark.parametrize("k", [8, 32])
def test_pcg_multi_rhs_matches_single(problem, k):
    P, ctx, f, orc = problem
    ctx.set_opts(precision=R.PREC_FP64, tol=1e-8, stop_rule=R.STOP_RELRES)
    B = np.stack([zero_sum_normal(P.ns, 100 + c) for c in range(k)], axis=1)
    X, info = ctx.pcg_solve(f, B)
    assert info["converged"] and info["relres_true"] <= 1e-8
    for c in [0, k // 2, k - 1]:
        x1, i1 = ctx.pcg_solve(f, B[:, c])
        np.testing.assert_allclose(X[:, c], x1, rtol=0, atol=1e-7 * np.abs(x1).max())


def test_fp32_mixed_reaches_fp64_residual(problem):
    P, ctx, f, orc = problem
    ctx.set_opts(precision=R.PREC_FP32_FACTOR, tol=1e-10, stop_rule=R.STOP_RELRES)
    b = zero_sum_normal(P.ns, 9)
    x, info = ctx.pcg_solve(f, b)
    assert info["converged"] and info["relres_true"] <= 1e-10


def test_pcg_without_graph(problem):
    P, ctx, f, orc = problem
    ctx.set_opts(precision=R.PREC_FP64, use_graph=0, tol=1e-6)
    b = zero_sum_normal(P.ns, 11)
    x, info = ctx.pcg_solve(f, b)
    ctx.set_opts(use_graph=1)
    x2, info2 = ctx.pcg_solve(f, b)
    assert info["iterations"] == info2["iterations"]
    np.testing.assert_array_equal(x, x2)  # same kernels, same order: identical bits


@pytest.mark.parametrize("precision", [R.PREC_FP64, R.PREC_FP32_FACTOR])
def test_pcg_bitwise_reproducible_across_factorizations(precision):
    """Two factorizations with one seed give bit-identical solves: the
    solve schedules (and so the order of every reduction) are independent
    of thread timing."""
    n, r, c, v, g = grid_laplacian((18, 17, 16), seed=31, excess_frac=0.05, wlo=1e-3, whi=1e3)
    b = None
    results = []
    for _ in range(2):
        ctx = R.Context(seed=8, precision=precision, tol=1e-8)
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        ns = f.info().n
        if b is None:
            b = zero_sum_normal(ns, 12)
        x, info = ctx.pcg_solve(f, b)
        results.append((x, info["iterations"], info["relres_true"]))
        f.free()
        ctx.close()
    assert results[0][1] == results[1][1]
    np.testing.assert_array_equal(results[0][0], results[1][0])
    assert results[0][2] == results[1][2]


def _hub_laplacian(leaves, seed):
    rng = np.random.default_rng(seed)
    n = leaves + 1
    a = np.concatenate([np.zeros(leaves, np.int64), np.arange(1, n)])
    b = np.concatenate([np.arange(1, n), np.roll(np.arange(1, n), -1)])
    w = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), len(a)))
    d = np.zeros(n)
    np.add.at(d, a, w)
    np.add.at(d, b, w)
    return (n, np.concatenate([a, b, np.arange(n)]).astype(np.int32),
            np.concatenate([b, a, np.arange(n)]).astype(np.int32), np.concatenate([-w, -w, d]))


@pytest.mark.parametrize("graph", ["power_law", "hub"])
def test_split_rows_match_oracle(graph):
    """Rows of L (power-law graph) or of L^T (hub ordered first) longer than
    the split threshold run as several part tasks; the preconditioner and
    PCG still match the oracle and repeat bit for bit."""
    if graph == "power_law":
        n, r, c, v, g = R.generate("chunglu", [20000, 150000, 2, 5000], wlo=1.0, whi=10.0, seed=7)
    else:
        (n, r, c, v), g = _hub_laplacian(3000, seed=3), False
    P = OracleProblem(n, r, c, v, trim=g)
    orc = P.factor(seed=12)
    rowlen = np.bincount(orc["rowind"], minlength=P.ns)
    collen = np.diff(orc["colptr"])
    assert max(rowlen.max(), collen.max()) > 1024
    ctx = R.Context(seed=12, precision=R.PREC_FP64, tol=1e-8)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        rr = zero_sum_normal(P.ns, 21)
        z = ctx.precond_apply(f, rr)
        ref = O.precond_apply(P.ns, orc["colptr"], orc["rowind"], orc["val"], orc["diag"], rr)
        np.testing.assert_allclose(z, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        np.testing.assert_array_equal(z, ctx.precond_apply(f, rr))
        x, info = ctx.pcg_solve(f, rr)
        xo, io = P.pcg(orc, rr, tol=1e-8)
        assert info["converged"] and abs(info["iterations"] - io["iterations"]) <= 1
        x2, info2 = ctx.pcg_solve(f, rr)
        np.testing.assert_array_equal(x, x2)
        f.free()
    finally:
        ctx.close()


def test_split_counters_recover_after_timeout():
    """A wait limit far below an apply's duration abandons the passes with
    some split rows' part counters part-way; the next apply with a normal
    limit must still match the oracle (the counters are cleared per call)."""
    n, r, c, v, g = R.generate("chunglu", [20000, 150000, 2, 5000], wlo=1.0, whi=10.0, seed=7)
    P = OracleProblem(n, r, c, v, trim=g)
    orc = P.factor(seed=12)
    assert np.bincount(orc["rowind"], minlength=P.ns).max() > 1024  # split rows exist
    ctx = R.Context(seed=12, precision=R.PREC_FP64, tol=1e-8)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        rr = zero_sum_normal(P.ns, 22)
        ref = O.precond_apply(P.ns, orc["colptr"], orc["rowind"], orc["val"], orc["diag"], rr)
        ctx.set_opts(timeout_s=1e-7)
        timeouts = 0
        for _ in range(4):
            try:
                ctx.precond_apply(f, rr)
            except R.RcholError as e:
                assert e.status == 5
                timeouts += 1
            try:
                ctx.pcg_solve(f, rr)
            except R.RcholError as e:
                assert e.status == 5
                timeouts += 1
        assert timeouts > 0
        ctx.set_opts(timeout_s=30.0)
        z = ctx.precond_apply(f, rr)
        np.testing.assert_allclose(z, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        x, info = ctx.pcg_solve(f, rr)
        assert info["converged"]
        f.free()
    finally:
        ctx.close()


def test_laplacian_without_ground():
    n, r, c, v, g = grid_laplacian((64, 64), seed=31)
    P = OracleProblem(n, r, c, v)
    ctx = R.Context(seed=2)
    try:
        ctx.set_triplets(n, r, c, v)
        f = ctx.factor()
        b = O.zero_sum_vector(n, 0)
        x, info = ctx.pcg_solve(f, b)
        xo, io = P.pcg(P.factor(seed=2), b, tol=1e-6)
        assert info["converged"] and abs(info["iterations"] - io["iterations"]) <= 1
        f.free()
    finally:
        ctx.close()


def test_timeout_is_reported_not_hung(problem):
    """A wait limit far below a solve's duration: the kernels give up,
    report RCHOL_ERR_TIMEOUT, and the context keeps working."""
    P, ctx, f, orc = problem
    ctx.set_opts(precision=R.PREC_FP64, timeout_s=1e-7, tol=1e-6)
    b = zero_sum_normal(P.ns, 13)
    with pytest.raises(R.RcholError) as e:
        ctx.pcg_solve(f, b)
    assert e.value.status == 5
    ctx.set_opts(timeout_s=30.0)
    x, info = ctx.pcg_solve(f, b)
    assert info["converged"]


def test_prepare_and_solve_drop_in(problem):
    """solver.hpp:236 signature on device arrays (torch owns the memory)."""
    import torch
    P, ctx, f, orc = problem
    dev = torch.device("cuda:0")
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    # reference factor format: CSR of L^T with the unit diagonal first in each row
    rows_ptr = [0]
    cols, vals = [], []
    for j in range(P.ns):
        s, e = orc["colptr"][j], orc["colptr"][j + 1]
        cols += [j] + list(orc["rowind"][s:e])
        vals += [1.0] + list(orc["val"][s:e])
        rows_ptr.append(len(cols))
    lap = [t(P.acp, torch.int32), t(P.arow, torch.int32), t(P.aval, torch.float64)]
    fac = [t(rows_ptr, torch.int32), t(vals, torch.float64), t(cols, torch.int32)]
    dg = t(orc["diag"], torch.float64)
    x = torch.zeros(P.ns, dtype=torch.float64, device=dev)
    info = R.prepare_and_solve(P.ns, lap[0].data_ptr(), lap[1].data_ptr(), lap[2].data_ptr(), fac[0].data_ptr(),
                               fac[1].data_ptr(), fac[2].data_ptr(), dg.data_ptr(), 1e-7, physics=True,
                               x_out=x.data_ptr())
    b = O.zero_sum_vector(P.ns, 0)
    xo, io = P.pcg(orc, b, tol=1e-7, max_iter=300, stop_rule=O.STOP_PRECOND)
    assert abs(info["iterations"] - io["iterations"]) <= 1
    np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=0, atol=1e-6 * np.abs(xo).max())


@pytest.mark.parametrize("dims", [(7, 9, 11), (16, 16, 24)])
def test_sliced_ell_spmv_matches_csr(dims):
    """The one-RHS PCG on the sliced-ELL copy of A (ragged last slice for
    7x9x11) against the CSR SpMV: q and p agree bit for bit, only the p.q
    partial sums follow another grid, so a few iterations agree to rounding
    and the converged solves to the tolerance."""
    n, r, c, v, g = grid_laplacian(dims, seed=41, excess_frac=0.05, wlo=1e-3, whi=1e3)
    out = {}
    for layout in (R.SPMV_AUTO, R.SPMV_CSR):
        ctx = R.Context(seed=3, precision=R.PREC_FP32_FACTOR, tol=1e-8, spmv_layout=layout)
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        ns = f.info().n
        b = zero_sum_normal(ns, 5)
        x, info = ctx.pcg_solve(f, b)
        ctx.set_opts(max_iter=3)
        x3, _ = ctx.pcg_solve(f, b)
        out[layout] = (x, info, x3)
        f.free()
        ctx.close()
    (xa, ia, a3), (xc, ic, c3) = out[R.SPMV_AUTO], out[R.SPMV_CSR]
    assert ia["converged"] and ic["converged"]
    assert abs(ia["iterations"] - ic["iterations"]) <= 1
    np.testing.assert_allclose(a3, c3, rtol=1e-12, atol=1e-12 * np.abs(c3).max())
    assert np.linalg.norm(xa - xc) <= 1e-6 * np.linalg.norm(xc)


def test_solver_kept_across_factors():
    """A context keeps its PCG solver (vectors and captured graph) when the
    factor changes: solves alternating between two live factors, and one
    after a factor is released and another made, equal those of a fresh
    context bit for bit."""
    n, r, c, v, g = grid_laplacian((14, 15, 13), seed=43, excess_frac=0.05, wlo=1e-2, whi=1e2)

    def fresh():
        ctx = R.Context(seed=6, precision=R.PREC_FP32_FACTOR, tol=1e-8)
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        return ctx

    ref_ctx = fresh()
    f = ref_ctx.factor()
    b = zero_sum_normal(f.info().n, 9)
    x_ref, i_ref = ref_ctx.pcg_solve(f, b)
    f.free()
    ref_ctx.close()

    ctx = fresh()
    f1 = ctx.factor()
    f2 = ctx.factor()  # other buffers, so the graph arguments change
    for f in (f1, f2, f1):
        x, info = ctx.pcg_solve(f, b)
        assert info["iterations"] == i_ref["iterations"]
        np.testing.assert_array_equal(x, x_ref)
    f1.free()
    f2.free()
    f3 = ctx.factor()  # reuses a released factor's buffers
    x, info = ctx.pcg_solve(f3, b)
    np.testing.assert_array_equal(x, x_ref)
    f3.free()

    # a new matrix of the same shape (the solver, trimmed matrix and
    # sliced-ELL copy keep their buffers) against a fresh context
    v2 = v * 2.5
    xs = []
    for c_ in (ctx, fresh()):
        c_.set_triplets(n, r, c, v2, trim_ground=g)
        f = c_.factor()
        xs.append(c_.pcg_solve(f, b)[0])
        f.free()
        c_.close()
    np.testing.assert_array_equal(xs[0], xs[1])


def test_hop_latency_floor():
    """The store -> poll hop between two SMs that bounds the sync-free
    solves from below: a finite positive time of the order of an L2 round
    trip, and a solve of depth d takes at least d of them."""
    ctx = R.Context()
    try:
        ns, sms = ctx.hop_latency(2048)
        assert 20.0 < ns < 20000.0
        assert all(s >= 0 for s in sms)
        with pytest.raises(R.RcholError):
            ctx.hop_latency(8)
        n, r, c, v, g = grid_laplacian((24, 24, 24), seed=3, excess_frac=0.05)
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        fi = f.info()
        assert fi.solve_depth > 1 and fi.solve_depth_b > 1
        ms = ctx.profile_solve(f, 1, reps=3)
        assert ms[1] * 1e6 >= fi.solve_depth * ns * 0.5
        assert ms[2] * 1e6 >= fi.solve_depth_b * ns * 0.5
        f.free()
    finally:
        ctx.close()


@pytest.mark.parametrize("precision,graph", [(R.PREC_FP64, "grid"), (R.PREC_FP32_FACTOR, "grid"),
                                             (R.PREC_FP32_FACTOR, "power_law")])
def test_backward_head_matches_persistent_kernel(precision, graph):
    """The first backward levels solved by the one-CTA head kernel: the
    factor of a 3-D grid (a few dozen narrow levels) and of a power-law
    graph (hundreds) gets a head, and PCG with it reaches the same iterate
    as with the head switched off (same z bit for bit; only the grouping of
    the r.z sum differs)."""
    if graph == "grid":
        n, r, c, v, g = grid_laplacian((20, 22, 24), seed=45, excess_frac=0.05, wlo=1e-2, whi=1e2)
    else:
        n, r, c, v, g = R.generate("chunglu", [60000, 600000, 2, 6000], wlo=1.0, whi=10.0, seed=11)
    out = {}
    for head in (1, 0):
        ctx = R.Context(seed=4, precision=precision, tol=1e-8, bwd_head=head)
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        fi = f.info()
        b = zero_sum_normal(fi.n, 11)
        x, info = ctx.pcg_solve(f, b)
        ctx.set_opts(max_iter=2)
        x2, _ = ctx.pcg_solve(f, b)
        out[head] = (fi.bwd_head_levels, fi.bwd_head_rows, x, info, x2)
        f.free()
        ctx.close()
    (hl, hr, xh, ih, x2h), (nl, nr, xn, inn, x2n) = out[1], out[0]
    assert hl >= 8 and hr > 0 and nl == 0 and nr == 0
    assert ih["converged"] and inn["converged"]
    assert abs(ih["iterations"] - inn["iterations"]) <= 1
    np.testing.assert_allclose(x2h, x2n, rtol=0, atol=1e-12 * np.abs(x2n).max())
    assert np.linalg.norm(xh - xn) <= 1e-7 * np.linalg.norm(xn)


def test_multi_rhs_layouts_built_on_first_use():
    """A factor's multi-RHS layouts (its rows copied in schedule order) are
    built on its first k > 1 apply or solve; before that the k > 1 sweeps
    read L's rows by row id.  Both forms sum the same entries in the same
    order: the allocation-free apply gives the same bits before and after."""
    torch = pytest.importorskip("torch")
    n, r, c, v, g = grid_laplacian((18, 16, 14), seed=47, excess_frac=0.05)
    ctx = R.Context(seed=5, precision=R.PREC_FP32_FACTOR)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        ns = f.info().n
        k = 4
        Rh = np.random.default_rng(9).standard_normal((ns, k))
        dev = torch.device("cuda", 0)
        Rd = torch.from_numpy(Rh).to(dev).contiguous()
        stream = torch.cuda.current_stream().cuda_stream
        out = []
        for step in range(2):
            Zd = torch.full((ns, k), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            ctx.precond_apply_noalloc(f, Rd.data_ptr(), Zd.data_ptr(), k, True, stream)
            torch.cuda.synchronize()
            out.append(Zd.cpu().numpy())
            if step == 0:
                ref = ctx.precond_apply(f, Rh, fp32=True)  # builds the layouts
        assert np.array_equal(out[0], out[1])
        np.testing.assert_allclose(out[1], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        f.free()
    finally:
        ctx.close()


def test_disconnected_graph_with_isolated_vertex():
    """Two grid components of different sizes and one vertex with no edges
    (zero degree, D = 0), in one ascending-degree order: the factor is
    bit-exact, and PCG on a right-hand side with zero sum on every component
    converges like the oracle's and leaves the isolated vertex at 0."""
    n, r, c, vals, iso, comp1, comp2 = disconnected_laplacian()
    P = OracleProblem(n, r, c, vals)
    orc = P.factor(seed=9)
    ctx = R.Context(seed=9)
    try:
        ctx.set_triplets(n, r, c, vals)
        f = ctx.factor()
        cp, ri, val, d = f.to_host()
        assert np.array_equal(cp, orc["colptr"]) and np.array_equal(ri, orc["rowind"])
        assert np.array_equal(val, orc["val"]) and np.array_equal(d, orc["diag"])
        assert d[iso] == 0.0
        b = per_component_rhs(n, comp1, comp2)
        x, info = ctx.pcg_solve(f, b)
        xo, io = P.pcg(orc, b, tol=1e-6)
        assert info["status"] == 0 and info["converged"] and info["relres_true"] <= 1e-6
        assert abs(info["iterations"] - io["iterations"]) <= 1
        assert x[iso] == 0.0
        f.free()
    finally:
        ctx.close()
