"""The allocation-free preconditioner apply (rchol_precond_apply_noalloc)
against the allocating one (rchol_precond_apply) on the same factor.

Both run the same sweeps over the same factor, so they agree to 1e-12
relative (FP64 and FP32 factor copies alike); the results are also checked
against the oracle's CPU apply on the host copy of the factor.  Two calls in a row check that
the shared scratch is reset between calls, and device free memory must not
move across a call.  This file is collected last so that it also runs after
every other GPU test in the same process.
"""
import numpy as np
import pytest

import pyoracle as O
import rchol_b200 as R

pytestmark = pytest.mark.gpu

LIMIT = 1 << 22  # n * k limit of the allocation-free scratch


@pytest.fixture(scope="module")
def setup():
    torch = pytest.importorskip("torch")
    n, r, c, v, g = R.generate("grid3d", [20, 20, 20], wlo=1e-2, whi=1e2, log_weights=True, seed=77)
    ctx = R.Context(seed=4, precision=R.PREC_FP32_FACTOR)
    ctx.set_triplets(n, r, c, v, trim_ground=g)
    f = ctx.factor()
    yield torch, ctx, f, n - 1 if g else n
    f.free()
    ctx.close()


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("k", [1, 8])
def test_noalloc_matches_precond_apply(setup, k, fp32):
    torch, ctx, f, ns = setup
    rng = np.random.default_rng(100 + k + int(fp32))
    Rs = [rng.standard_normal((ns, k)) for _ in range(2)]
    refs = [ctx.precond_apply(f, Rh if k > 1 else Rh[:, 0], fp32=fp32).reshape(ns, k) for Rh in Rs]
    dev = torch.device("cuda", 0)
    Rd = [torch.from_numpy(Rh).to(dev).contiguous() for Rh in Rs]  # row-major n x k
    Zd = [torch.full((ns, k), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    ctx.precond_apply_noalloc(f, Rd[0].data_ptr(), Zd[0].data_ptr(), k, fp32, stream)
    free_before = torch.cuda.mem_get_info(0)[0]
    ctx.precond_apply_noalloc(f, Rd[1].data_ptr(), Zd[1].data_ptr(), k, fp32, stream)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free_before
    for z, ref in zip(Zd, refs):
        got = z.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    # and directly against the oracle's L^-T D^+ L^-1 on the same factor
    # (FP64 sweeps: 1e-12; the FP32 factor copy: 2e-5, as the other tests)
    cp, ri, lv, d = f.to_host()
    tol = 2e-5 if fp32 else 1e-12
    for z, Rh in zip(Zd, Rs):
        got = z.cpu().numpy()
        for c in range(k):
            ref = O.precond_apply(ns, cp, ri, lv, d, Rh[:, c])
            np.testing.assert_allclose(got[:, c], ref, rtol=tol, atol=tol * np.abs(ref).max())


def test_noalloc_rejects_oversize_and_bad_k():
    torch = pytest.importorskip("torch")
    # 52^3 = 140608 > 2^22 / 32 unknowns: k = 32 is over the limit, k = 16 is not
    n, r, c, v, g = R.generate("grid3d", [52, 52, 52], seed=78)
    ctx = R.Context(seed=4)
    try:
        ctx.set_triplets(n, r, c, v, trim_ground=g)
        f = ctx.factor()
        ns = n - 1 if g else n
        assert ns * 32 > LIMIT >= ns * 16
        Rd = torch.zeros((ns, 32), dtype=torch.float64, device="cuda")
        Zd = torch.zeros_like(Rd)
        with pytest.raises(R.RcholError, match="allocation-free limit"):
            ctx.precond_apply_noalloc(f, Rd.data_ptr(), Zd.data_ptr(), 32)
        with pytest.raises(R.RcholError):
            ctx.precond_apply_noalloc(f, Rd.data_ptr(), Zd.data_ptr(), 3)
        # the largest admissible block for this n still runs
        R16 = torch.from_numpy(np.random.default_rng(5).standard_normal((ns, 16))).cuda()
        Z16 = torch.zeros_like(R16)
        ctx.precond_apply_noalloc(f, R16.data_ptr(), Z16.data_ptr(), 16)
        ref = ctx.precond_apply(f, R16.cpu().numpy())
        np.testing.assert_allclose(Z16.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
        f.free()
    finally:
        ctx.close()
