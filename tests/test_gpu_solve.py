"""GPU parity of the two-surface operator, right-hand side and GMRES solve
(2S/main.cpp:140-677) against the reference's golden outputs and the oracle."""
import numpy as np
import pytest

import highreg
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plan16(ctx, g2s):
    p = highreg.Plan2S(ctx, g2s, mode=highreg.HR_TREE, P=int(g2s["P"]), N0=int(g2s["N0"]), theta=0.6)
    yield p
    p.close()


def test_plan_lifecycle_around_the_background_batch(ctx, g2s):
    # the FP64 stresslet batch is segmented on a host thread of its own after
    # creation: destroying a plan at once joins it; the right-hand side runs
    # beside it; the work counts and the first matvec wait for it
    opt = dict(mode=highreg.HR_TREE, P=int(g2s["P"]), N0=int(g2s["N0"]), theta=0.6)
    for _ in range(3):
        highreg.Plan2S(ctx, g2s, **opt).close()
    p = highreg.Plan2S(ctx, g2s, **opt)
    b = p.rhs(g2s["f0"], g2s["f1"])
    assert rel_err(b, g2s["rhs"]) < 1e-12
    assert p.work(0)["direct_pairs_near"] > 0
    assert rel_err(p.matvec(g2s["mv_u"]), g2s["mv_y"]) < 1e-12
    p.close()


def test_matvec_matches_reference(plan16, g2s):
    y = plan16.matvec(g2s["mv_u"])
    assert rel_err(y, g2s["mv_y"]) < 1e-12


def test_rhs_matches_reference(plan16, g2s):
    b = plan16.rhs(g2s["f0"], g2s["f1"])
    assert rel_err(b, g2s["rhs"]) < 1e-12


def test_solve_matches_reference(plan16, g2s):
    b = plan16.rhs(g2s["f0"], g2s["f1"])
    x, rep = plan16.solve(b, restart=15, tol=1e-10)
    ref_hist = g2s["sol_hist"]
    assert rep["iterations"] == len(ref_hist)
    assert np.allclose(rep["resid_hist"], ref_hist, rtol=1e-4)
    assert rel_err(x, g2s["sol_x"]) < 1e-9


def test_solution_satisfies_system_under_oracle_operator(plan16, g2s, oracle):
    """Size-independent property: the GPU solution x satisfies A x = b with the
    oracle's own operator, to the solve tolerance."""
    sc = oracle.scene(g2s, tree=True, P=int(g2s["P"]), N0=int(g2s["N0"]))
    b = oracle.rhs_2s(sc, g2s["f0"], g2s["f1"])
    x, rep = plan16.solve(b, restart=50, tol=1e-10)
    r = b - oracle.matvec_2s(sc, x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10


def test_warm_start_and_guess_rejection(plan16, g2s):
    b = plan16.rhs(g2s["f0"], g2s["f1"])
    x, rep = plan16.solve(b, restart=50, tol=1e-10)
    # a good guess converges in fewer iterations to the same answer
    x2, rep2 = plan16.solve(b, x0=x + 1e-6 * np.sin(np.arange(len(x))), restart=50, tol=1e-10)
    assert rep2["iterations"] < rep["iterations"] and not rep2["guess_rejected"]
    assert rel_err(x2, x) < 1e-8
    # a guess worse than zero is dropped (falls back to the zero guess)
    x3, rep3 = plan16.solve(b, x0=1e3 * np.ones(len(x)), restart=50, tol=1e-10)
    assert rep3["guess_rejected"] == 1
    assert rel_err(x3, x) < 1e-8


def test_iteration_cap_reports_not_converged(plan16, g2s):
    b = plan16.rhs(g2s["f0"], g2s["f1"])
    with pytest.raises(highreg.HrError) as e:
        plan16.solve(b, restart=15, tol=1e-10, max_iter=3)
    assert e.value.code == highreg.HR_ERR_NOT_CONVERGED


def test_h32_direct_and_tree_operators_vs_oracle(ctx, oracle):
    G = highreg.Geometry2S(32).scene
    rng = np.random.default_rng(11)
    u = rng.standard_normal(3 * (len(G["area0"]) + len(G["area1"])))
    for mode in (highreg.HR_DIRECT, highreg.HR_TREE):
        plan = highreg.Plan2S(ctx, G, mode=mode, P=6, N0=1000, theta=0.6)
        sc = oracle.scene(G, tree=mode == highreg.HR_TREE, P=6, N0=1000)
        assert rel_err(plan.matvec(u), oracle.matvec_2s(sc, u)) < 1e-12
        assert rel_err(plan.rhs(G["f0"], G["f1"]), oracle.rhs_2s(sc, G["f0"], G["f1"])) < 1e-12
        w = plan.work(0)
        assert w["direct_pairs_near"] + w["direct_pairs_far"] > 0 and w["flops"] > 0
        if mode == highreg.HR_TREE:
            assert w["proxy_pairs"] > 0
        plan.close()


def test_h32_solve_golden_history(ctx):
    """Reference h = 1/32 (P = 6, N0 = 1000): 13 iterations to 7.8214e-11."""
    G = highreg.Geometry2S(32).scene
    plan = highreg.Plan2S(ctx, G, mode=highreg.HR_TREE, P=6, N0=1000, theta=0.6)
    b = plan.rhs(G["f0"], G["f1"])
    x, rep = plan.solve(b, restart=15, tol=1e-10)
    assert rep["iterations"] == 13
    assert abs(rep["residual"] - 7.8214e-11) / 7.8214e-11 < 1e-3
    plan.close()
