"""CUDA factor (through the C-ABI) against the oracle, bit-exact.

The GPU eliminates vertices in whatever order the ready queue serves them;
with Philox uniforms keyed by (seed, vertex, slot) and total orders for the
merge and the value sort, the factor must equal the oracle's ORC_MODE_B200
factor exactly: same pattern, same FP64 bits in L and D.
"""
import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R
from helpers import OracleProblem, grid_laplacian, zero_sum_normal

pytestmark = pytest.mark.gpu

CASES = {
    "grid32_logw": dict(dims=(32, 32), seed=1),
    "grid40_unit": dict(dims=(40, 40), seed=2, log_weights=False),
    "cube10_sddm": dict(dims=(10, 10, 10), seed=3, excess_frac=0.05, wlo=1e-3, whi=1e3),
    "cube24_logw": dict(dims=(24, 24, 24), seed=4, wlo=1e-3, whi=1e3),
    # every row has a diagonal excess: the ground column holds 5,833 entries,
    # more than one warp counts (the grid-wide long-column count)
    "cube18_ground_all": dict(dims=(18, 18, 18), seed=6, excess_frac=1.0, wlo=1e-3, whi=1e3),
}


def _gpu_factor(n, r, c, v, trim, seed, **opts):
    ctx = R.Context(seed=seed, **opts)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=trim)
        f = ctx.factor()
        out = f.to_host()
        info = f.info()
        f.free()
        return out, info
    finally:
        ctx.close()


def _compare(gpu, orc):
    cp, ri, val, d = gpu
    assert np.array_equal(cp, orc["colptr"])
    assert np.array_equal(ri, orc["rowind"])
    assert np.array_equal(val, orc["val"])  # bit-exact FP64
    assert np.array_equal(d, orc["diag"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_factor_bitexact_vs_oracle(name):
    spec = dict(CASES[name])
    dims = spec.pop("dims")
    seed = spec.pop("seed")
    n, r, c, v, ground = grid_laplacian(dims, seed=seed, **spec)
    P = OracleProblem(n, r, c, v, trim=ground)
    orc = P.factor(seed=seed + 100)
    gpu, info = _gpu_factor(n, r, c, v, ground, seed + 100)
    _compare(gpu, orc)
    assert info.nnz_strict == orc["stats"]["nnz_strict"] or ground
    assert info.attempts >= 1


def test_factor_config1_bitexact():
    n, r, c, v, g = R.generate("grid2d", [256, 256], seed=0)
    P = OracleProblem(n, r, c, v)
    orc = P.factor(seed=1)
    gpu, info = _gpu_factor(n, r, c, v, False, 1)
    _compare(gpu, orc)
    assert info.fills == orc["stats"]["fills"]


@pytest.mark.parametrize("opts", [dict(warps_per_block=1, num_blocks=1), dict(num_blocks=64),
                                  dict(bucket_cap=1, slab_entries=32), dict(bucket_cap=2, pool_mult=1.0)])
def test_factor_independent_of_launch_shape_and_pools(opts):
    """One warp, a few warps, tiny buckets (overflow chunks), tiny shared
    slabs (global slab path), a tiny pool (capacity retry): same bits."""
    n, r, c, v, _ = grid_laplacian((20, 20, 6), seed=5, wlo=1e-3, whi=1e3)
    P = OracleProblem(n, r, c, v)
    orc = P.factor(seed=7)
    gpu, info = _gpu_factor(n, r, c, v, False, 7, **opts)
    _compare(gpu, orc)
    if opts.get("bucket_cap", 32) <= 2:
        assert info.overflow_fills > 0 and info.chunks_used > 0
    if opts.get("slab_entries", 256) == 32:
        assert info.big_vertices > 0
    if opts.get("pool_mult", 6.0) == 1.0:
        assert info.attempts >= 1


def _hub_laplacian(leaves, seed):
    """Vertex 0 joined to every leaf, leaves joined in a ring: in natural
    order vertex 0 gathers all `leaves` entries at once."""
    rng = np.random.default_rng(seed)
    n = leaves + 1
    a = np.concatenate([np.zeros(leaves, np.int64), np.arange(1, n)])
    b = np.concatenate([np.arange(1, n), np.roll(np.arange(1, n), -1)])
    w = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), len(a)))
    d = np.zeros(n)
    np.add.at(d, a, w)
    np.add.at(d, b, w)
    rows = np.concatenate([a, b, np.arange(n)]).astype(np.int32)
    cols = np.concatenate([b, a, np.arange(n)]).astype(np.int32)
    vals = np.concatenate([-w, -w, d])
    return n, rows, cols, vals


def test_factor_large_gather_uses_shared_slab():
    """A gather larger than the per-warp scratch (4096 entries) runs in one
    of the shared slabs and stays bit-exact."""
    n, r, c, v = _hub_laplacian(6000, seed=5)
    P = OracleProblem(n, r, c, v, trim=False)
    gpu, info = _gpu_factor(n, r, c, v, False, seed=6)
    _compare(gpu, P.factor(seed=6))
    assert info.max_gather >= 6000


def _multi_hub_laplacian(leaves, hubs, seed):
    """Leaves 0..leaves-1 each joined to every hub (numbered last): every
    leaf elimination samples fills between hubs, so the hub columns gather
    thousands of duplicates of a few rows."""
    rng = np.random.default_rng(seed)
    n = leaves + hubs
    a = np.repeat(np.arange(leaves), hubs)
    b = np.tile(np.arange(leaves, n), leaves)
    w = np.exp(rng.uniform(np.log(1e-2), np.log(1e2), len(a)))
    d = np.zeros(n)
    np.add.at(d, a, w)
    np.add.at(d, b, w)
    rows = np.concatenate([a, b, np.arange(n)]).astype(np.int32)
    cols = np.concatenate([b, a, np.arange(n)]).astype(np.int32)
    vals = np.concatenate([-w, -w, d])
    return n, rows, cols, vals


@pytest.mark.parametrize("leaves,hubs", [(3000, 4), (1500, 12)])
def test_factor_long_duplicate_runs_bitexact(leaves, hubs):
    """Runs of one row longer than a lane orders in registers are ordered
    by value and added by the whole warp; the factor equals the oracle's
    bit for bit."""
    n, r, c, v = _multi_hub_laplacian(leaves, hubs, seed=21)
    P = OracleProblem(n, r, c, v, trim=False)
    gpu, info = _gpu_factor(n, r, c, v, False, seed=22)
    _compare(gpu, P.factor(seed=22))
    assert info.max_gather > 1000


@pytest.mark.parametrize("opts", [dict(), dict(bucket_cap=2, slab_entries=32)])
def test_factor_power_law_bitexact(opts):
    """Power-law graph: hub columns take long overflow chunk chains and
    gathers in global slabs (radix-sorted, searched through the shared
    index); the factor still equals the oracle's bit for bit."""
    n, r, c, v, g = R.generate("chunglu", [6000, 30000, 2, 1500], wlo=1.0, whi=10.0, seed=7)
    P = OracleProblem(n, r, c, v, trim=g)
    gpu, info = _gpu_factor(n, r, c, v, g, seed=12, **opts)
    _compare(gpu, P.factor(seed=12))
    assert info.max_gather > 256


def test_factor_repeatable_in_one_context():
    n, r, c, v, _ = grid_laplacian((30, 30), seed=8)
    ctx = R.Context(seed=3)
    try:
        ctx.set_triplets(n, r, c, v)
        a = ctx.factor()
        b = ctx.factor()
        A, B = a.to_host(), b.to_host()
        for x, y in zip(A, B):
            assert np.array_equal(x, y)
        a.free()
        b.free()
    finally:
        ctx.close()


def test_factor_write_read_roundtrip(tmp_path):
    n, r, c, v, g = grid_laplacian((9, 9, 9), seed=9, excess_frac=0.1)
    ctx = R.Context(seed=2)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        prefix = str(tmp_path) + "/"
        f.write(prefix)
        f2 = ctx.factor_read(prefix)
        A, B = f.to_host(), f2.to_host()
        assert np.array_equal(A[0], B[0]) and np.array_equal(A[1], B[1])
        np.testing.assert_allclose(A[2], B[2], rtol=1e-15)
        np.testing.assert_array_equal(A[3], B[3])
        # the file is the reference's format: unit diagonal, rows >= cols, 1-based
        rows, cols, vals, diag = O.read_factor_files(prefix, f.info().n)
        assert np.all(rows >= cols) and np.all(vals[rows == cols] == 1.0)
    finally:
        ctx.close()


def test_invalid_inputs_report_status():
    ctx = R.Context()
    try:
        with pytest.raises(R.RcholError) as e:
            ctx.factor()
        assert e.value.status == 9
        n, r, c, v, _ = grid_laplacian((4, 4), seed=1)
        v = v.copy()
        v[0] = np.inf
        with pytest.raises(R.RcholError):
            ctx.set_triplets(n, r, c, v)
    finally:
        ctx.close()


def test_bad_colptr_is_rejected_on_the_device():
    """set_csc checks colptr (starts at 0, never decreases, ends at nnz) on
    the device after the upload; a bad one reports RCHOL_ERR_INVALID and
    leaves the context without a matrix, and a good one loads after it."""
    n, r, c, v, _ = grid_laplacian((6, 5), seed=2)
    cp, ri, val = R.csc_from_triplets(n, r, c, v)
    ctx = R.Context()
    try:
        bad = cp.copy()
        bad[3], bad[4] = bad[4], bad[3]
        with pytest.raises(R.RcholError) as e:
            ctx.set_csc(n, bad, ri, val)
        assert e.value.status == 1
        with pytest.raises(R.RcholError) as e:
            ctx.factor()
        assert e.value.status == 9
        ctx.set_csc(n, cp, ri, val)
        f = ctx.factor()
        assert f.info().n == n
        f.free()
    finally:
        ctx.close()


def test_factor_timeout_is_reported_then_recovers():
    """A wait limit far below the elimination's queue waits: the factor
    kernel gives up with RCHOL_ERR_TIMEOUT (bounded device waits, no hang),
    and the next factorization with the normal limit is bit-exact."""
    n, r, c, v, g = grid_laplacian((40, 40, 40), seed=9, excess_frac=0.05)
    P = OracleProblem(n, r, c, v, trim=g)
    orc = P.factor(seed=5)
    ctx = R.Context(seed=5)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        ctx.set_opts(timeout_s=1e-7)
        timeouts = 0
        for _ in range(3):
            try:
                ctx.factor().free()
            except R.RcholError as e:
                assert e.status == 5
                timeouts += 1
        assert timeouts > 0
        ctx.set_opts(timeout_s=30.0)
        f = ctx.factor()
        cp, ri, val, d = f.to_host()
        assert np.array_equal(cp, orc["colptr"]) and np.array_equal(ri, orc["rowind"])
        assert np.array_equal(val, orc["val"]) and np.array_equal(d, orc["diag"])
        f.free()
    finally:
        ctx.close()


def test_factor_outlives_its_context():
    """A factor freed after its context (as on an error path that skips the
    factor's release) is detached by rchol_destroy: its host copy still
    works and freeing it does not touch the destroyed context."""
    n, r, c, v, g = grid_laplacian((20, 20), seed=5)
    P = OracleProblem(n, r, c, v, trim=g)
    orc = P.factor(seed=6)
    ctx = R.Context(seed=6)
    ctx.set_triplets(n, r, c, v, trim_ground=g)
    f = ctx.factor()
    ctx.close()
    cp, ri, val, d = f.to_host()
    assert np.array_equal(ri, orc["rowind"]) and np.array_equal(val, orc["val"])
    f.free()


@pytest.mark.parametrize("case,tail", [("powerlaw", 400), ("powerlaw", 6000), ("cube_sddm", 10 ** 9)])
def test_cooperative_tail_is_bit_exact(case, tail):
    """The last `tail` vertices eliminated one at a time by a whole CTA
    (CTA radix sorts, chained Kogge-Stone carries) give the oracle's factor
    bit for bit, including a tail that covers every vertex."""
    if case == "powerlaw":
        n, r, c, v, g = R.generate("chunglu", [6000, 30000, 2, 1500], wlo=1.0, whi=10.0, seed=7)
    else:
        n, r, c, v, g = grid_laplacian((11, 10, 9), seed=3, excess_frac=0.05, wlo=1e-3, whi=1e3)
    P = OracleProblem(n, r, c, v, trim=g)
    orc = P.factor(seed=21)
    ctx = R.Context(seed=21, tail_vertices=min(tail, n))
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        assert f.info().tail_vertices == min(tail, n)
        cp, ri, val, d = f.to_host()
        assert np.array_equal(cp, orc["colptr"]) and np.array_equal(ri, orc["rowind"])
        assert np.array_equal(val, orc["val"]) and np.array_equal(d, orc["diag"])
        b = zero_sum_normal(P.ns, 4)
        x, info = ctx.pcg_solve(f, b)
        assert info["converged"]
        f.free()
    finally:
        ctx.close()


def test_autotune_choices_are_used_and_cached():
    """rchol_autotune profiles the gathers, keeps only choices that time
    faster, writes them into the context's options (the next factorization
    reports the chosen tail) and serves a second call from its cache."""
    n, r, c, v, g = R.generate("chunglu", [20000, 150000, 2, 5000], wlo=1.0, whi=10.0, seed=7)
    ctx = R.Context(seed=3, precision=R.PREC_FP32_FACTOR)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        t1 = ctx.autotune(max_rhs=32)
        assert not t1["from_cache"] and t1["max_gather"] > 32
        assert t1["rhs_block"] in (1, 2, 4, 8, 16, 32) and t1["bucket_cap"] in (8, 16, 32, 64, 128)
        assert t1["ms_factor_tuned"] <= t1["ms_factor_default"]
        assert all(x > 0 for x in t1["per_rhs_ms"])
        assert ctx.opts.tail_vertices == t1["tail_vertices"] and ctx.opts.rhs_block == t1["rhs_block"]
        f = ctx.factor()
        assert f.info().tail_vertices == t1["tail_vertices"]
        f.free()
        t2 = ctx.autotune(max_rhs=32)
        assert t2["from_cache"] and t2["tail_vertices"] == t1["tail_vertices"]
        # a k-RHS solve runs in blocks of the chosen width and still converges
        B = np.random.default_rng(2).standard_normal((n - (1 if g else 0), 32))
        B -= B.mean(axis=0)
        f = ctx.factor()
        X, info = ctx.pcg_solve(f, B)
        assert info["converged"]
        f.free()
    finally:
        ctx.close()
