"""GPU parity of the boundary sums against the reference's golden outputs and
the oracle, through the C ABI.

Tolerance (FP64 path): max |gpu - ref| <= 1e-12 * max |ref|. The GPU sums
contract multiply-adds into FMAs and add the same terms in a different order
than the reference; nothing else differs.
"""
import numpy as np
import pytest

from conftest import rel_err
import e2g_util

pytestmark = pytest.mark.gpu
TOL = 1e-12
PAIRS = [(0, 0), (0, 1), (1, 0), (1, 1)]


def _surf(g, s):
    return g["xq%d" % s], g["nrm%d" % s], g["area%d" % s]


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("s,t", PAIRS)
def test_stokeslet_sums(ctx, g2s, s, t, mode):
    DEL, P, N0 = float(g2s["DEL"]), int(g2s["P"]), int(g2s["N0"])
    xq, nrm, area = _surf(g2s, s)
    f = g2s["f%d" % s]
    opt = dict(mode=mode, P=P, N0=N0, theta=0.6)
    if s == t:
        out = ctx.sl_onsurf(DEL, xq, nrm, area, f, ctr=g2s["ctr%d" % s], **opt)
    else:
        out = ctx.sl_offsurf(DEL, xq, nrm, area, f, g2s["xq%d" % t], g2s["b%d" % t], g2s["n0%d" % t],
                             g2s["f0%d" % t], ctr=g2s["ctr%d" % s], **opt)
    assert rel_err(out, g2s["sl_t%d_%d%d" % (mode, s, t)]) < TOL


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("s,t", PAIRS)
def test_stresslet_sums(ctx, g2s, s, t, mode):
    DEL, P, N0 = float(g2s["DEL"]), int(g2s["P"]), int(g2s["N0"])
    xq, nrm, area = _surf(g2s, s)
    g = g2s["g%d" % s]
    opt = dict(mode=mode, P=P, N0=N0, theta=0.6)
    if s == t:
        out = ctx.dl_onsurf(DEL, xq, nrm, area, g, ctr=g2s["ctr%d" % s], **opt)
    else:
        out = ctx.dl_offsurf(DEL, xq, nrm, area, g, g2s["xq%d" % t], g2s["b%d" % t], g2s["x0%d" % t],
                             g2s["n0%d" % t], g2s["g0interp%d" % t], ctr=g2s["ctr%d" % s], **opt)
    assert rel_err(out, g2s["dl_t%d_%d%d" % (mode, s, t)]) < TOL


@pytest.mark.parametrize("t", [0, 1])
def test_density_interpolation(ctx, g2s, t):
    s = 1 - t
    g0 = ctx.interpolate_dl_density(float(g2s["h"]), g2s["xq%d" % s], g2s["g%d" % s], g2s["ctr%d" % s],
                                    g2s["plane%d" % s], g2s["x0%d" % t], g2s["nrst%d" % t], g2s["i123%d" % t])
    assert rel_err(g0, g2s["g0interp%d" % t]) < 1e-14


def test_tree_h32_random_density_vs_oracle(ctx, oracle):
    """A second geometry (h = 1/32, P = 6, N0 = 1000) and seeded random densities."""
    import highreg

    G = highreg.Geometry2S(32).scene
    rng = np.random.default_rng(7)
    DEL = G["DEL"]
    for s, t in PAIRS:
        xq, nrm, area = _surf(G, s)
        g = rng.standard_normal(len(xq))
        if s == t:
            ref, _ = oracle.kitc(2, 6, 1000, 0.6, G["ctr%d" % s], DEL, xq, nrm, area, g)
            out = ctx.dl_onsurf(DEL, xq, nrm, area, g, ctr=G["ctr%d" % s], mode=1, P=6, N0=1000)
        else:
            g0 = rng.standard_normal(len(G["xq%d" % t]))
            ref, _ = oracle.kitc(3, 6, 1000, 0.6, G["ctr%d" % s], DEL, xq, nrm, area, g, xt=G["xq%d" % t],
                                 b=G["b%d" % t], x0=G["x0%d" % t], n0=G["n0%d" % t], dens0=g0)
            out = ctx.dl_offsurf(DEL, xq, nrm, area, g, G["xq%d" % t], G["b%d" % t], G["x0%d" % t],
                                 G["n0%d" % t], g0, ctr=G["ctr%d" % s], mode=1, P=6, N0=1000)
        assert rel_err(out, ref) < TOL


def test_e2g_sums(ctx, ge2g):
    N, h, DEL = int(ge2g["N"]), float(ge2g["h"]), float(ge2g["DEL"])
    xq, nrm, area, f = ge2g["xq"], ge2g["nrm"], ge2g["area"], ge2g["f"]
    M = N + 1
    xt, gi = e2g_util.face_targets(N, h)
    assert rel_err(ctx.e2g_p_away(xq, area, f, xt), ge2g["p_faces"][gi]) < TOL
    u = ctx.e2g_sl_away(xq, area, f, xt)
    uf = ge2g["u_faces"].reshape(3, M ** 3)
    ref = np.stack([uf[k][gi] for k in range(3)], 1).ravel()
    assert rel_err(u, ref) < TOL
    xs, bs, x0s, n0s, f0s, gb = e2g_util.band_targets(N, h, ge2g["nrst"], ge2g["b"], ge2g["x0"], ge2g["n0"])
    assert rel_err(ctx.e2g_p_7ord(DEL, xq, nrm, area, f, xs, bs, f0s, n0s), ge2g["p_band"][gb]) < TOL
    ub = ctx.e2g_sl_7ord(DEL, xq, nrm, area, f, xs, bs, f0s, n0s)
    uband = ge2g["u_band"].reshape(3, M ** 3)
    ref = np.stack([uband[k][gb] for k in range(3)], 1).ravel()
    assert rel_err(ub, ref) < TOL


def test_empty_and_ragged_inputs(ctx, g2s):
    DEL = float(g2s["DEL"])
    xq, nrm, area = _surf(g2s, 0)
    # empty target set
    out = ctx.sl_offsurf(DEL, xq, nrm, area, g2s["f0"], np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0))
    assert out.shape == (0,)
    # a ragged count (not a multiple of the 128-target block) matches the direct oracle
    n = 301
    f = g2s["f0"]
    out = ctx.sl_offsurf(DEL, xq, nrm, area, f, g2s["xq1"][:3 * n], g2s["b1"][:n], g2s["n01"][:3 * n],
                         g2s["f01"][:3 * n], mode=0)
    ref = g2s["sl_t0_01"][:3 * n]
    assert rel_err(out, ref) < TOL


def test_nan_input_rejected(ctx, g2s):
    import highreg

    geo = dict(g2s)
    geo["xq0"] = geo["xq0"].copy()
    geo["xq0"][5] = np.nan
    with pytest.raises(highreg.HrError) as e:
        highreg.Plan2S(ctx, geo, mode=1, P=4, N0=300)
    assert e.value.code == highreg.HR_ERR_NAN
