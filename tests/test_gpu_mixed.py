"""Mixed precision (FP32 far field with FP64 per-target accumulation, FP64
near-surface pairs): error against the FP64 path and the relaxed GMRES.

Tolerances: a mixed operator application is within 3e-5 (max-norm, relative)
of the FP64 one (FP32 rounding of individual terms, amplified by cancellation
between terms of both signs); a mixed solve reaches the same 1e-10 relative residual,
checked with an FP64 operator, and its solution agrees with the FP64
solution to 1e-8."""
import numpy as np
import pytest
import torch

import highreg
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def geo32():
    return highreg.Geometry2S(32).scene


@pytest.fixture(scope="module")
def plan32(ctx, geo32):
    p = highreg.Plan2S(ctx, geo32, mode=highreg.HR_TREE, P=6, N0=1000, theta=0.6)
    yield p
    p.close()


def test_mixed_operator_error(plan32):
    n = plan32.n
    u = torch.tensor(np.random.default_rng(2).standard_normal(n), dtype=torch.float64, device="cuda")
    y64 = torch.zeros_like(u)
    y32 = torch.zeros_like(u)
    plan32.matvec_dev(u, y64, highreg.HR_FP64)
    plan32.matvec_dev(u, y32, highreg.HR_MIXED)
    torch.cuda.synchronize()
    e = rel_err(y32.cpu().numpy(), y64.cpu().numpy())
    print('mixed operator max-norm relative error', e)
    assert 0 < e < 3e-5, e


def test_mixed_single_sums(ctx, geo32):
    g = geo32
    DEL = g["DEL"]
    for mode in (highreg.HR_DIRECT, highreg.HR_TREE):
        a = ctx.sl_offsurf(DEL, g["xq0"], g["nrm0"], g["area0"], g["f0"], g["xq1"], g["b1"], g["n01"], g["f01"],
                           ctr=g["ctr0"], mode=mode, P=6, N0=1000)
        b = ctx.sl_offsurf(DEL, g["xq0"], g["nrm0"], g["area0"], g["f0"], g["xq1"], g["b1"], g["n01"], g["f01"],
                           ctr=g["ctr0"], mode=mode, P=6, N0=1000, precision=highreg.HR_MIXED)
        assert rel_err(b, a) < 3e-5
        a = ctx.dl_onsurf(DEL, g["xq1"], g["nrm1"], g["area1"], g["f1"], ctr=g["ctr1"], mode=mode, P=6, N0=1000)
        b = ctx.dl_onsurf(DEL, g["xq1"], g["nrm1"], g["area1"], g["f1"], ctr=g["ctr1"], mode=mode, P=6, N0=1000,
                          precision=highreg.HR_MIXED)
        assert rel_err(b, a) < 3e-5


def test_mixed_solve_reaches_fp64_residual(plan32, geo32):
    b = plan32.rhs(geo32["f0"], geo32["f1"])
    x64, r64 = plan32.solve(b, restart=50, tol=1e-10, true_residual=True)
    x32, r32 = plan32.solve(b, restart=50, tol=1e-10, precision=highreg.HR_MIXED)
    assert r32["matvecs_mixed"] > 0
    assert r32["true_residual"] <= 1e-9
    assert r64["true_residual"] <= 1e-9
    assert rel_err(x32, x64) < 1e-8


def test_fp32_operator_error(plan32):
    """All pairs in FP32 (r < 1e-14 limits excepted): the off-surface
    smoothing brackets cancel for close pairs, so the error is at least the
    mixed mode's (equal when the worst entry comes from the on-surface and far
    field terms the two modes share) and stays bounded; the refined solve
    below absorbs it."""
    n = plan32.n
    u = torch.tensor(np.random.default_rng(2).standard_normal(n), dtype=torch.float64, device="cuda")
    y64 = torch.zeros_like(u)
    y32 = torch.zeros_like(u)
    ym = torch.zeros_like(u)
    plan32.matvec_dev(u, y64, highreg.HR_FP64)
    plan32.matvec_dev(u, y32, highreg.HR_FP32)
    plan32.matvec_dev(u, ym, highreg.HR_MIXED)
    torch.cuda.synchronize()
    e32 = rel_err(y32.cpu().numpy(), y64.cpu().numpy())
    em = rel_err(ym.cpu().numpy(), y64.cpu().numpy())
    print('FP32 operator max-norm relative error', e32, 'mixed', em)
    assert em <= e32 < 1e-3


def test_fp32_solve_reaches_fp64_residual(plan32, geo32):
    b = plan32.rhs(geo32["f0"], geo32["f1"])
    x64, _ = plan32.solve(b, restart=50, tol=1e-10)
    x32, r32 = plan32.solve(b, restart=50, tol=1e-10, precision=highreg.HR_FP32)
    assert r32["matvecs_mixed"] > 0
    assert r32["true_residual"] <= 1e-9
    assert rel_err(x32, x64) < 1e-8


def test_inner_tree_solve_reaches_fp64_residual(ctx, geo32):
    """GMRES-IR whose inner cycles run on a coarser treecode (P = 4, N0 = 300):
    the FP64 true residual, taken with the plan's own treecode, still meets the
    tolerance, and the solution matches the all-FP64 one to 1e-8."""
    p = highreg.Plan2S(ctx, geo32, mode=highreg.HR_TREE, P=6, N0=1000, theta=0.6)
    b = p.rhs(geo32["f0"], geo32["f1"])
    x64, r64 = p.solve(b, restart=50, tol=1e-10, true_residual=True)
    u = np.random.default_rng(5).standard_normal(p.n)
    ym = torch.zeros(p.n, dtype=torch.float64, device="cuda")
    yi = torch.zeros_like(ym)
    ut = torch.tensor(u, dtype=torch.float64, device="cuda")
    p.matvec_dev(ut, ym, highreg.HR_MIXED)
    acc = p.set_inner_tree(4, 300, 0.6)
    p.matvec_dev(ut, yi, highreg.HR_MIXED)
    torch.cuda.synchronize()
    e_inner = rel_err(yi.cpu().numpy(), ym.cpu().numpy())
    print("inner-treecode operator vs the plan's (mixed):", e_inner)
    assert 0 < e_inner < 1e-2  # P = 4 against P = 6: ~2e-3 at h = 1/32
    # the measured relative L2 error on the fixed density (the solve's default accuracy)
    assert 0 < acc <= e_inner * 10
    xi, ri = p.solve(b, restart=50, tol=1e-10, precision=highreg.HR_MIXED)
    print("inner-treecode solve:", ri["iterations"], "iterations,", ri["matvecs_fp64"], "FP64 matvecs")
    assert ri["matvecs_mixed"] > 0
    assert ri["true_residual"] <= 1e-10
    assert rel_err(xi, x64) < 1e-8
    # its work, counted from its interaction lists
    w = p.work(2)
    assert w["direct_pairs_near"] > 0 and w["proxy_pairs"] > 0 and w["moment_terms"] > 0
    # removing it restores the plan's own operator
    assert p.set_inner_tree(0, 0) == 0.0
    with pytest.raises(highreg.HrError):
        p.work(2)
    p.matvec_dev(ut, yi, highreg.HR_MIXED)
    torch.cuda.synchronize()
    assert rel_err(yi.cpu().numpy(), ym.cpu().numpy()) == 0.0
    p.close()


@pytest.mark.parametrize("P,N0", [(6, 1000), (10, 2000), (4, 300)])
def test_tensor_core_upward_pass_matches_fp64(ctx, geo32, P, N0):
    """The 3xTF32 tcgen05 upward pass (reduced-precision operator) against the
    FP64 one: split TF32 products with FP32 accumulation keep ~1e-6 relative
    accuracy per node and channel."""
    plan = highreg.Plan2S(ctx, geo32, mode=highreg.HR_TREE, P=P, N0=N0, theta=0.6)
    x = np.random.default_rng(5).standard_normal(plan.n)
    e = plan.check_upward_pass(x)
    print("upward pass, P=%d: max relative difference %.3e" % (P, e))
    assert 0 < e < 2e-5
    plan.close()
