"""Warm-start host side on the CPU: seeded instances, features, the rigid-motion
property the instances' right-hand side relies on, and the MLP oracle's own
finite-difference pin. No GPU calls."""
import os
import struct
import sys

import numpy as np
import pytest

import highreg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle  # noqa: E402

SEED = 20261203


def _ellipsoid(inst, s):
    a = np.array(inst.geom.axes[:])
    c = np.array(inst.geom.center[s][:])
    R = np.array(inst.geom.unrot[s][:]).reshape(3, 3) if inst.geom.rotated[s] else np.eye(3)
    return a, c, R


def test_instances_are_seeded_and_in_range():
    seen = []
    for i in range(12):
        w = highreg.warm_instance(SEED, i)
        w2 = highreg.warm_instance(SEED, i)
        assert w.as_dict() == w2.as_dict()
        assert 0.04 <= w.gap <= 0.6
        assert abs(np.linalg.norm(w.U[:]) - 1) < 1e-12 and abs(np.linalg.norm(w.Omega[:]) - 1) < 1e-12
        R = np.array(w.geom.unrot[1][:]).reshape(3, 3)
        assert np.abs(R @ R.T - np.eye(3)).max() < 1e-12 and abs(np.linalg.det(R) - 1) < 1e-12
        seen.append(w.gap)
    assert len(set(seen)) == len(seen)
    assert highreg.warm_instance(SEED + 1, 0).gap != seen[0]


@pytest.mark.parametrize("index", [0, 3, 7])
def test_instance_gap_is_the_distance_between_the_solids(index):
    """Dense sampling of surface 2 against the exact distance to surface 1."""
    w = highreg.warm_instance(SEED, index)
    a1, c1, R1 = _ellipsoid(w, 0)
    a2, c2, R2 = _ellipsoid(w, 1)
    th, ph = np.meshgrid(np.linspace(0, np.pi, 401), np.linspace(0, 2 * np.pi, 801), indexing="ij")
    body = np.stack([a2[0] * np.cos(th), a2[1] * np.sin(th) * np.cos(ph), a2[2] * np.sin(th) * np.sin(ph)], -1)
    pts = c2 + body.reshape(-1, 3) @ R2  # world = c + R^T body
    # distance of each sample to ellipsoid 1 by the Lagrange root t of
    # sum (a_i v_i / (t + a_i^2))^2 = 1, solved by vectorized bisection
    v = (pts - c1) @ R1.T
    assert ((v / a1) ** 2).sum(1).min() > 1.0
    lo = np.zeros(len(v))
    hi = np.linalg.norm(v, axis=1) * a1.max()
    for _ in range(100):
        t = 0.5 * (lo + hi)
        F = ((a1 * v / (t[:, None] + a1 ** 2)) ** 2).sum(1) - 1
        lo = np.where(F > 0, t, lo)
        hi = np.where(F > 0, hi, t)
    x = a1 ** 2 * v / ((0.5 * (lo + hi))[:, None] + a1 ** 2)
    d = np.linalg.norm(v - x, axis=1).min()
    assert w.gap <= d + 1e-9
    assert d - w.gap < 2e-4  # sampling error of the grid on surface 2


def test_features_match_independent_formulas():
    w = highreg.warm_instance(SEED, 2)
    geo = highreg.Geometry2S(16, w.geom).scene
    F, u = highreg.warm_features(geo, w)
    n0 = len(geo["area0"])
    assert F.shape == (n0 + len(geo["area1"]), 12)
    xyz = np.concatenate([geo["xq0"], geo["xq1"]]).reshape(-1, 3)
    nrm = np.concatenate([geo["nrm0"], geo["nrm1"]]).reshape(-1, 3)
    rot = highreg.warm_frames(w)
    assert np.array_equal(rot[0], np.eye(3))
    assert np.array_equal(rot[1], np.array(w.geom.unrot[1][:]).reshape(3, 3))
    body = np.concatenate([nrm[:n0] @ rot[0].T, nrm[n0:] @ rot[1].T])
    assert np.abs(F[:, 0:3] - body).max() < 1e-6
    # principal curvatures: eigenvalues of the shape operator of the level set,
    # computed here with numpy's symmetric eigensolver
    for s, sl in ((0, slice(0, n0)), (1, slice(n0, None))):
        a, c0, R = _ellipsoid(w, s)
        body = (xyz[sl] - c0) @ R.T
        A, C = a[1], a[0]  # equatorial and polar semi-axes (polar along body x)
        g = 2 * body / a ** 2
        Hs = np.diag(2 / a ** 2)
        gn = np.linalg.norm(g, axis=1)
        nn = g / gn[:, None]
        k1s, k2s = [], []
        for i in range(len(body)):
            P = np.eye(3) - np.outer(nn[i], nn[i])
            S = P @ Hs @ P / gn[i]
            ev = np.sort(np.linalg.eigvalsh(S))
            k1s.append(ev[2])
            k2s.append(ev[1])
        assert np.abs(F[sl, 3] - np.array(k1s)).max() < 1e-5 * 4
        assert np.abs(F[sl, 4] - np.array(k2s)).max() < 1e-5 * 4
        # the mean curvature agrees with the reference's spheroid formula
        cos_sq = (body[:, 1] ** 2 + body[:, 2] ** 2) / A ** 2
        temp = A * A + (C * C - A * A) * cos_sq
        H_ref = C * (A * A + temp) / (2 * A * np.sqrt(temp ** 3))
        assert np.abs(0.5 * (F[sl, 3] + F[sl, 4]) - H_ref).max() < 1e-4
        # distance to the other surface equals the generator's signed distance
        b = geo["b%d" % s]
        ok = geo["nrst%d" % s] > 0
        assert ok.sum() > 100
        assert np.abs(F[sl, 5][ok] - b[ok]).max() < 1e-6
        dirn = F[sl, 6:9]
        assert np.abs(np.linalg.norm(dirn, axis=1) - 1).max() < 1e-6
        x0 = geo["x0%d" % s].reshape(-1, 3)
        want = (x0 - xyz[sl]) / np.linalg.norm(x0 - xyz[sl], axis=1)[:, None]
        assert np.abs(dirn[ok] - want[ok] @ rot[s].T).max() < 1e-5
    r = xyz - np.array(w.xmid[:])
    uu = np.array(w.U[:]) + np.cross(np.array(w.Omega[:]), r)
    assert np.abs(u.reshape(-1, 3) - uu).max() < 1e-14
    ub = np.concatenate([uu[:n0] @ rot[0].T, uu[n0:] @ rot[1].T])
    assert np.abs(F[:, 9:12] - ub).max() < 1e-6


def test_body_frame_tension_matches_the_reference_law_for_the_default_scene():
    """The reference's second surface is turned about z only, so the body-frame
    tension gives the reference's force bit for bit."""
    p = highreg.Geometry2S.default_params()
    a = highreg.Geometry2S(16, p).scene
    p.tension_body = 1
    b = highreg.Geometry2S(16, p).scene
    for s in (0, 1):
        assert np.array_equal(a["f%d" % s], b["f%d" % s])
        assert np.array_equal(a["f0%d" % s], b["f0%d" % s])


def test_rigid_motion_is_an_eigenfunction_of_the_operator(oracle):
    """(I - 2/3 D) u = 2/3 u for a rigid motion u on both closed surfaces, so the
    instances' right-hand side rhs(f) + 2/3 u has solution u + A^-1 rhs(f)."""
    w = highreg.warm_instance(SEED, 5)
    geo = highreg.Geometry2S(16, w.geom).scene
    _, u = highreg.warm_features(geo, w)
    sc = oracle.scene(geo, tree=False)
    Au = oracle.matvec_2s(sc, u)
    assert np.abs(Au - (2.0 / 3.0) * u).max() / np.abs(u).max() < 2e-3


def test_mlp_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.standard_normal(mlp_oracle.NPARAMS) * 0.2
    X = rng.standard_normal((40, 12))
    T = rng.standard_normal((40, 3))
    mean, std, sc = rng.standard_normal(12) * 0.1, 0.5 + rng.random(12), 1.7
    loss, g = mlp_oracle.loss_and_grad(p, X, T, mean, std, sc)
    idx = rng.choice(mlp_oracle.NPARAMS, 60, replace=False)
    eps = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += eps
        lp, _ = mlp_oracle.loss_and_grad(q, X, T, mean, std, sc)
        q[k] -= 2 * eps
        lm, _ = mlp_oracle.loss_and_grad(q, X, T, mean, std, sc)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-7 + 1e-5 * abs(g[k])


def test_committed_weights_file_is_well_formed():
    path = os.path.join(ROOT, "high-order-regularization_b200", "data", "warmstart_h64.hrmlp")
    if not os.path.exists(path):
        pytest.skip("no trained weights committed")
    raw = open(path, "rb").read()
    assert raw[:8] == b"HRMLP001"
    assert struct.unpack("<5i", raw[8:28]) == (12, 64, 64, 64, 3)
    assert len(raw) == 8 + 20 + 4 * 25 + 4 * 9347 + 8
    h = 1469598103934665603
    for byte in raw[:-8]:
        h = ((h ^ byte) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    assert struct.unpack("<Q", raw[-8:])[0] == h
    params = np.frombuffer(raw[128:128 + 4 * 9347], np.float32)
    assert np.isfinite(params).all()
