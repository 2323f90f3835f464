"""Pins the oracle (oracle/highreg_oracle.c) to the reference's own outputs.

The golden fixtures were produced by the unmodified reference
(tests/golden/make_golden.py); the C restatement must reproduce them bit for
bit (it follows the reference's operation order and is built without FMA).
"""
import numpy as np
import pytest

from conftest import rel_err
import e2g_util


def _surf(g, s):
    return g["xq%d" % s], g["nrm%d" % s], g["area%d" % s]


PAIRS = [(0, 0), (0, 1), (1, 0), (1, 1)]


@pytest.mark.parametrize("s,t", PAIRS)
def test_sl_direct_and_tree(oracle, g2s, s, t):
    DEL, P, N0 = float(g2s["DEL"]), int(g2s["P"]), int(g2s["N0"])
    xq, nrm, area = _surf(g2s, s)
    f = g2s["f%d" % s]
    if s == t:
        d = oracle.sl_onsurf_direct(DEL, xq, nrm, area, f)
        tr, _ = oracle.kitc(0, P, N0, 0.6, g2s["ctr%d" % s], DEL, xq, nrm, area, f)
    else:
        d = oracle.sl_offsurf_direct(DEL, xq, nrm, area, f, g2s["xq%d" % t], g2s["b%d" % t],
                                     g2s["f0%d" % t], g2s["n0%d" % t])
        tr, _ = oracle.kitc(1, P, N0, 0.6, g2s["ctr%d" % s], DEL, xq, nrm, area, f, xt=g2s["xq%d" % t],
                            b=g2s["b%d" % t], n0=g2s["n0%d" % t], dens0=g2s["f0%d" % t])
    assert np.array_equal(d, g2s["sl_t0_%d%d" % (s, t)])
    assert np.array_equal(tr, g2s["sl_t1_%d%d" % (s, t)])


@pytest.mark.parametrize("s,t", PAIRS)
def test_dl_direct_and_tree(oracle, g2s, s, t):
    DEL, P, N0 = float(g2s["DEL"]), int(g2s["P"]), int(g2s["N0"])
    xq, nrm, area = _surf(g2s, s)
    g = g2s["g%d" % s]
    if s == t:
        d = oracle.dl_onsurf_direct(DEL, xq, nrm, area, g)
        tr, _ = oracle.kitc(2, P, N0, 0.6, g2s["ctr%d" % s], DEL, xq, nrm, area, g)
    else:
        g0 = g2s["g0interp%d" % t]
        d = oracle.dl_offsurf_direct(DEL, xq, nrm, area, g, g2s["xq%d" % t], g2s["b%d" % t],
                                     g2s["x0%d" % t], g2s["n0%d" % t], g0)
        tr, _ = oracle.kitc(3, P, N0, 0.6, g2s["ctr%d" % s], DEL, xq, nrm, area, g, xt=g2s["xq%d" % t],
                            b=g2s["b%d" % t], x0=g2s["x0%d" % t], n0=g2s["n0%d" % t], dens0=g0)
    assert np.array_equal(d, g2s["dl_t0_%d%d" % (s, t)])
    assert np.array_equal(tr, g2s["dl_t1_%d%d" % (s, t)])


@pytest.mark.parametrize("t", [0, 1])
def test_density_interpolation(oracle, g2s, t):
    s = 1 - t
    g0 = oracle.interp_dl_density(float(g2s["h"]), g2s["ctr%d" % s], g2s["xq%d" % s], g2s["g%d" % s],
                                  g2s["nrst%d" % t], g2s["x0%d" % t], g2s["i123%d" % t])
    assert np.array_equal(g0, g2s["g0interp%d" % t])


def test_matvec_rhs_solve(oracle, g2s):
    sc = oracle.scene(g2s, tree=True, P=int(g2s["P"]), N0=int(g2s["N0"]))
    assert np.array_equal(oracle.matvec_2s(sc, g2s["mv_u"]), g2s["mv_y"])
    b = oracle.rhs_2s(sc, g2s["f0"], g2s["f1"])
    assert np.array_equal(b, g2s["rhs"])
    x, hist = oracle.gmres_2s(sc, b, im=15)
    ref_hist = g2s["sol_hist"]
    assert len(hist) == len(ref_hist)
    # the reference prints residuals with 6 significant digits
    assert np.allclose(hist, ref_hist, rtol=1e-5, atol=0)
    assert np.array_equal(x, g2s["sol_x"])


def test_e2g_sums(oracle, ge2g):
    N, h, DEL = int(ge2g["N"]), float(ge2g["h"]), float(ge2g["DEL"])
    xq, nrm, area, f = ge2g["xq"], ge2g["nrm"], ge2g["area"], ge2g["f"]
    M = N + 1
    xt, gi = e2g_util.face_targets(N, h)
    p = oracle.e2g_p_away(xq, area, f, xt)
    assert np.array_equal(p, ge2g["p_faces"][gi])
    u = oracle.e2g_sl_away(xq, area, f, xt)
    uf = ge2g["u_faces"].reshape(3, M ** 3)
    for k in range(3):
        assert np.array_equal(u[k::3], uf[k][gi])
    bt = e2g_util.band_targets(N, h, ge2g["nrst"], ge2g["b"], ge2g["x0"], ge2g["n0"])
    xs, bs, x0s, n0s, f0s, gb = bt
    pb = oracle.e2g_p_7ord(DEL, xq, nrm, area, f, xs, bs, f0s, n0s)
    assert np.array_equal(pb, ge2g["p_band"][gb])
    ub = oracle.e2g_sl_7ord(DEL, xq, nrm, area, f, xs, bs, f0s, n0s)
    uband = ge2g["u_band"].reshape(3, M ** 3)
    for k in range(3):
        assert np.array_equal(ub[k::3], uband[k][gb])


def test_e2g_poisson(oracle, ge2g):
    N, h = int(ge2g["N"]), float(ge2g["h"])
    b2, out = e2g_util.masks(N, h, ge2g["nrst"], ge2g["band2"])
    p_ext = oracle.solve_poisson(N, 3.0, h, b2, out, ge2g["p_band"], ge2g["p_band"], 0)
    # the reference's DST is the stand-in's O(n^4) sum: same algorithm and order
    assert rel_err(p_ext, ge2g["p_ext"]) < 1e-13
    M = N + 1
    ub = ge2g["u_band"].reshape(3, M ** 3)
    ue = ge2g["u_ext"].reshape(3, M ** 3)
    for v in range(3):
        uu = oracle.solve_poisson(N, 3.0, h, b2, out, ge2g["p_ext"], ub[v], v + 1)
        assert rel_err(uu, ue[v]) < 1e-13


def test_dst_poisson(oracle, ge2g):
    n = int(ge2g["N"]) - 1
    out = oracle.dst_poisson(n, ge2g["dst_in"])
    assert rel_err(out, ge2g["dst_out"]) < 1e-13


def test_dst_is_involution_up_to_scale(oracle):
    # RODFT00 applied twice is 2(n+1) times the identity on each axis
    n = 9
    a = np.random.default_rng(3).standard_normal(n ** 3)
    b = oracle.dst1_3d(n, oracle.dst1_3d(n, a))
    assert rel_err(b / (2 * (n + 1)) ** 3, a) < 1e-13


def _ref_or_skip(name):
    import os

    import oracle as oracle_mod

    if not os.path.exists(os.path.join(oracle_mod.REF_DIR, name)):
        pytest.skip("reference build %s not present" % name)
    return oracle_mod


def test_reference_scene_loader_and_sampled_sums(g2s):
    """The reference program driven from loaded arrays (ref2s_load) and on a
    target sample (ref2s_sample_eval) reproduces its own full direct sums and
    nearest-point densities of the fixture bit for bit."""
    om = _ref_or_skip("libref2s_P4_N300.so")
    R = om.Ref2S(4, 300)
    R.load(g2s, g=[g2s["g0"], g2s["g1"]])
    for s, t in PAIRS:
        n = len(g2s["area%d" % t])
        idx = np.arange(n, dtype=np.int32)[::-1].copy()  # every target, in reverse order
        sl, _ = R.sample_eval(0, s, t, idx)
        assert np.array_equal(sl.reshape(-1, 3), g2s["sl_t0_%d%d" % (s, t)].reshape(-1, 3)[idx])
        dl, g0 = R.sample_eval(1, s, t, idx)
        assert np.array_equal(dl.reshape(-1, 3), g2s["dl_t0_%d%d" % (s, t)].reshape(-1, 3)[idx])
        if s != t:
            assert np.array_equal(g0.reshape(-1, 3), g2s["g0interp%d" % t].reshape(-1, 3)[idx])


def test_reference_e2g_loader_and_sampled_sums(ge2g):
    """The reference extend-to-grid program driven from loaded arrays
    (refe2g_load) reproduces its own band and face sums of the fixture, on the
    whole index grid and on a sample of it."""
    om = _ref_or_skip("librefe2g.so")
    N = int(ge2g["N"])
    M = N + 1
    R = om.RefE2G().load(N, ge2g)
    p = R.eval_p_band(R.eval_p_faces())
    assert np.array_equal(p, ge2g["p_band"])
    nrst = ge2g["nrst"]
    tagged = np.flatnonzero(nrst >= 0)
    sample = tagged[::7]
    keep = np.full_like(nrst, -1)
    keep[sample] = nrst[sample]
    R.set_nrst(keep)
    ps = R.eval_p_band(np.zeros(M ** 3))
    b = ge2g["b"]
    out = sample[(b[nrst[sample]] > 0.0) | (np.abs(b[nrst[sample]]) < 1e-12)]
    assert np.array_equal(ps[out], ge2g["p_band"][out])
    face = np.array([0, 5 * M + 3, M * M * N + 7 * M + 2, (M * M + M + 1) * N], dtype=np.int64)
    xyz = np.stack(np.unravel_index(face, (M, M, M)), axis=1).astype(np.float64) * float(ge2g["h"])
    u, pf = R.away_points(xyz.ravel())
    assert np.array_equal(pf, ge2g["p_faces"][face])
    uf = ge2g["u_faces"].reshape(3, -1)[:, face].T.ravel()
    assert np.array_equal(u, uf)
