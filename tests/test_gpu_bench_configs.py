"""GPU parity at the sizes the benchmark and the precision study run, against
the reference itself (the unmodified reference compiled into oracle/_ref):

* two-surface solve at h = 1/64, KITC P = 6, N0 = 2000 (the bench workload):
  right-hand side and operator element-wise against the reference's eval_SL /
  solve_IE_1step, the GMRES residual history and solution against the
  reference's own solve (fixture tests/golden/ref2s_N64_P6_N02000_sampled.npz,
  made by tests/golden/make_golden.py), and the reduced-precision operator and
  solves against the same reference values;
* two-surface sums at h = 1/256 (P = 10, N0 = 8000): a seeded sample of
  targets of every sum kind against the reference's direct sums (its
  eval_Stokes_*_offSurf drivers and per-target on-surface functions, with its
  interpolate_DL_density for the stresslet's nearest-point densities), for the
  GPU's direct sums (1e-12), its treecode (treecode tolerance) and its
  reduced-precision sums;
* extend-to-grid at N = 384: a seeded sample of band and box-face grid
  points against the reference's band drivers (eval_{u,p}_BI_nearSurfc on an
  index grid that keeps only the sample) and its plain sums, for the
  pipeline's FP64, mixed and FP32 sums.

Errors are max |gpu - ref| / max |ref| ("max") and ||gpu - ref||_2 /
||ref||_2 ("l2"); each test prints its table.
"""
import os

import numpy as np
import pytest

import highreg
from conftest import GOLDEN, rel_err

pytestmark = pytest.mark.gpu

oracle_mod = pytest.importorskip("oracle")


def _errs(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return (float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)),
            float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))


def _ref2s(P, N0):
    path = os.path.join(oracle_mod.REF_DIR, "libref2s_P%d_N%d.so" % (P, N0))
    if not os.path.exists(path):
        pytest.skip("reference build %s not present" % os.path.basename(path))
    return oracle_mod.Ref2S(P, N0)


# ------------------------------------------------------------ h = 1/64 (bench)
@pytest.fixture(scope="module")
def h64(ctx):
    geo = highreg.Geometry2S(64).scene
    plan = highreg.Plan2S(ctx, geo, mode=highreg.HR_TREE, P=6, N0=2000, theta=0.6)
    yield geo, plan
    plan.close()


@pytest.fixture(scope="module")
def g64():
    d = np.load(os.path.join(GOLDEN, "ref2s_N64_P6_N02000_sampled.npz"))
    return {k: d[k] for k in d.files}


def test_h64_geometry_matches_reference_bitwise(h64):
    geo, _ = h64
    R = _ref2s(6, 2000).setup(64)
    ref = R.geometry()
    for k, v in ref.items():
        if k in geo:
            assert np.array_equal(np.asarray(geo[k]), np.asarray(v)), k


def test_h64_rhs_and_operator_match_reference(h64, g64):
    """Element-wise against the reference's own eval_SL and solve_IE_1step at
    the bench's configuration (the live reference where it was built, and
    always its stored sample)."""
    geo, plan = h64
    n = plan.n
    idx = g64["idx"]
    u = np.random.default_rng(int(g64["mv_seed"])).standard_normal(n)
    b = plan.rhs(geo["f0"], geo["f1"])
    y = plan.matvec(u)
    assert rel_err(b[idx], g64["rhs"]) < 1e-12
    assert rel_err(y[idx], g64["mv_y"]) < 1e-12
    R = _ref2s(6, 2000).setup(64)
    b_ref = R.rhs()
    y_ref = R.matvec(u)
    eb, ey = _errs(b, b_ref), _errs(y, y_ref)
    print("h=1/64 FP64 rhs err max %.2e l2 %.2e; matvec err max %.2e l2 %.2e" % (eb + ey))
    assert eb[0] < 1e-12 and ey[0] < 1e-12
    # the reduced-precision operator (GMRES-IR's inner matvec) against the same reference values
    import torch

    xd = torch.tensor(u, dtype=torch.float64, device="cuda")
    yd = torch.zeros_like(xd)
    plan.matvec_dev(xd, yd, highreg.HR_MIXED)
    torch.cuda.synchronize()
    em = _errs(yd.cpu().numpy(), y_ref)
    print("h=1/64 mixed-precision matvec err max %.2e l2 %.2e" % em)
    assert em[0] < 3e-5


def test_h64_solve_matches_reference_history(h64, g64):
    """GMRES(15) to 1e-10 on the bench configuration: the reference's 13
    iterations to 6.19681e-11 and its residual history; its solution at the
    sampled unknowns. The reduced-precision solve reaches the same tolerance
    and the same solution."""
    geo, plan = h64
    idx = g64["idx"]
    hist = g64["sol_hist"]
    assert len(hist) == 13 and abs(hist[-1] - 6.19681e-11) / 6.19681e-11 < 1e-4
    b = plan.rhs(geo["f0"], geo["f1"])
    x, rep = plan.solve(b, restart=15, tol=1e-10)
    assert rep["iterations"] == len(hist)
    assert np.allclose(rep["resid_hist"], hist, rtol=1e-4)
    e64 = _errs(x[idx], g64["sol_x"])
    xm, rm = plan.solve(b, restart=50, tol=1e-10, precision=highreg.HR_MIXED)
    em = _errs(xm[idx], g64["sol_x"])
    print("h=1/64 solution vs reference: FP64 max %.2e l2 %.2e (%d it); mixed max %.2e l2 %.2e "
          "(true residual %.2e)" % (e64 + (rep["iterations"],) + em + (rm["true_residual"],)))
    assert e64[0] < 1e-9
    assert rm["true_residual"] <= 1e-10 and em[0] < 1e-8


# --------------------------------------------------------- h = 1/256 (sampled)
def _sample(rng, b, DEL, n_near, n_far):
    near = np.flatnonzero(np.abs(b) <= 8.0 * DEL)
    far = np.flatnonzero(np.abs(b) > 8.0 * DEL)
    pick = [rng.choice(near, min(n_near, len(near)), replace=False),
            rng.choice(far, min(n_far, len(far)), replace=False)]
    return np.sort(np.concatenate(pick)).astype(np.int32)


def _rows(v, idx):
    return v.reshape(-1, 3)[idx].ravel()


def test_h256_sampled_sums_match_reference_direct(ctx):
    """Every sum kind of the two-surface operator at h = 1/256 on a seeded
    sample of targets (near and far, both surfaces) against the reference's
    direct sums: the GPU's direct sums to 1e-12, its treecode (P = 10,
    N0 = 8000) to 1e-6, its reduced-precision treecode to 1e-4; the
    stresslet's nearest-point densities against the reference's
    interpolate_DL_density to 1e-12."""
    R = _ref2s(10, 8000)
    geo = highreg.Geometry2S(256).scene
    DEL, h = geo["DEL"], geo["h"]
    g = [geo["f0"], geo["f1"]]  # a smooth density for the stresslet sums: the interfacial force
    R.load(geo, g=g)
    rng = np.random.default_rng(256)
    tree = dict(mode=highreg.HR_TREE, P=10, N0=8000, theta=0.6)
    rows = []
    for s in (0, 1):
        xq, nrm, area, ctr = geo["xq%d" % s], geo["nrm%d" % s], geo["area%d" % s], geo["ctr%d" % s]
        # on-surface sums (targets = the surface's own points)
        idx = np.sort(rng.choice(len(area), 1500, replace=False)).astype(np.int32)
        for kind, name in ((0, "SL on"), (1, "DL on")):
            ref, _ = R.sample_eval(kind, s, s, idx)
            fn = ctx.sl_onsurf if kind == 0 else ctx.dl_onsurf
            got = {p: _rows(fn(DEL, xq, nrm, area, g[s], ctr=ctr, precision=p, **tree), idx)
                   for p in (highreg.HR_FP64, highreg.HR_MIXED)}
            got["direct"] = _rows(fn(DEL, xq, nrm, area, g[s], ctr=ctr, mode=highreg.HR_DIRECT), idx)
            rows.append((name, s, got, ref))
        # off-surface sums at the other surface's points
        t = 1 - s
        bt = geo["b%d" % t]
        idx = _sample(rng, bt, DEL, 1000, 500)
        ref, _ = R.sample_eval(0, s, t, idx)
        args = (DEL, xq, nrm, area, g[s], geo["xq%d" % t], bt, geo["n0%d" % t], geo["f0%d" % t])
        got = {p: _rows(ctx.sl_offsurf(*args, ctr=ctr, precision=p, **tree), idx)
               for p in (highreg.HR_FP64, highreg.HR_MIXED)}
        got["direct"] = _rows(ctx.sl_offsurf(*args, ctr=ctr, mode=highreg.HR_DIRECT), idx)
        rows.append(("SL off", s, got, ref))
        ref, g0_ref = R.sample_eval(1, s, t, idx)
        g0 = ctx.interpolate_dl_density(h, xq, g[s], ctr, geo["plane%d" % s], geo["x0%d" % t],
                                        geo["nrst%d" % t], geo["i123%d" % t])
        assert rel_err(_rows(g0, idx), g0_ref) < 1e-12
        args = (DEL, xq, nrm, area, g[s], geo["xq%d" % t], bt, geo["x0%d" % t], geo["n0%d" % t], g0)
        got = {p: _rows(ctx.dl_offsurf(*args, ctr=ctr, precision=p, **tree), idx)
               for p in (highreg.HR_FP64, highreg.HR_MIXED, highreg.HR_FP32)}
        got["direct"] = _rows(ctx.dl_offsurf(*args, ctr=ctr, mode=highreg.HR_DIRECT), idx)
        rows.append(("DL off", s, got, ref))
    names = {highreg.HR_FP64: "tree fp64", highreg.HR_MIXED: "tree mixed", highreg.HR_FP32: "tree fp32",
             "direct": "direct fp64"}
    print("h=1/256 sampled sums vs the reference's direct sums (max / l2):")
    for name, s, got, ref in rows:
        e = {k: _errs(v, ref) for k, v in got.items()}
        print("  %-6s surface %d: " % (name, s) + ", ".join("%s %.2e / %.2e" % ((names[k],) + e[k]) for k in e))
        assert e["direct"][0] < 1e-12
        assert e[highreg.HR_FP64][0] < 1e-6  # the treecode's own approximation error (P = 10, theta = 0.6)
        assert e[highreg.HR_MIXED][0] < 1e-4
        if highreg.HR_FP32 in e:
            assert e[highreg.HR_FP32][0] < 1e-4


# ------------------------------------------------------ E2G N = 384 (sampled)
def test_e2g_n384_sampled_grid_points_match_reference(ctx):
    """The pipeline's sums at N = 384 on a seeded sample of band grid points
    (outside or on the surface, where the reference's band drivers evaluate)
    and box-face grid points, against the reference's eval_u_BI_nearSurfc /
    eval_p_BI_nearSurfc (run on an index grid holding only the sample) and its
    plain sums stokes_SL_away / stokes_pressure_away; FP64 to 1e-12, mixed and
    FP32 to 1e-7."""
    N = 384
    M = N + 1
    e = highreg.E2G(ctx, N)
    sc = e.scene()
    R = oracle_mod.RefE2G()
    if not oracle_mod.ref_available():
        e.close()
        pytest.skip("reference build not present")
    R.load(N, sc)
    rng = np.random.default_rng(384)
    nrst = sc["nrst"]
    b = sc["b"]
    tagged = np.flatnonzero(nrst >= 0)
    outside = tagged[(b[nrst[tagged]] > 0.0) | (np.abs(b[nrst[tagged]]) < 1e-12)]
    ii, jj, kk = np.unravel_index(outside, (M, M, M))
    interior = outside[(ii > 0) & (ii < N) & (jj > 0) & (jj < N) & (kk > 0) & (kk < N)]
    band = np.sort(rng.choice(interior, 2000, replace=False))
    keep = np.full_like(nrst, -1)
    keep[band] = nrst[band]
    R.set_nrst(keep)
    zero = np.zeros(M ** 3)
    p_ref = R.eval_p_band(zero)[band]
    u_ref = np.stack([a[band] for a in R.eval_u_band([zero, zero, zero])], axis=1).ravel()
    # box faces: points on the six faces
    fi = rng.integers(0, M, size=(1500, 3))
    ax = rng.integers(0, 3, size=1500)
    fi[np.arange(1500), ax] = rng.integers(0, 2, size=1500) * N
    face = np.unique(np.ravel_multi_index((fi[:, 0], fi[:, 1], fi[:, 2]), (M, M, M)))
    fxyz = np.stack(np.unravel_index(face, (M, M, M)), axis=1).astype(np.float64) * (3.0 / N)
    uf_ref, pf_ref = R.away_points(fxyz.ravel())
    print("E2G N=384 sampled sums vs the reference (max / l2):")
    for prec, name, tol in ((highreg.HR_FP64, "fp64", 1e-12), (highreg.HR_MIXED, "mixed", 1e-7),
                            (highreg.HR_FP32, "fp32", 1e-7)):
        e.run(prec)
        p = e.get(0)
        u = e.get(1).reshape(3, -1)
        res = {"band p": _errs(p[band], p_ref),
               "band u": _errs(np.stack([u[k][band] for k in range(3)], axis=1).ravel(), u_ref),
               "face p": _errs(p[face], pf_ref),
               "face u": _errs(np.stack([u[k][face] for k in range(3)], axis=1).ravel(), uf_ref)}
        print("  %-5s " % name + ", ".join("%s %.2e / %.2e" % ((k,) + v) for k, v in res.items()))
        for k, v in res.items():
            assert v[0] < tol, (name, k, v)
    e.close()
