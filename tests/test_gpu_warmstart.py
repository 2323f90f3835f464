"""The warm-start network's CUDA kernels against the FP64 numpy oracle, and
what the trained network gains over the method without it. All calls go
through the C ABI (libhighreg_b200.so)."""
import os
import sys

import numpy as np
import pytest
import torch

import highreg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "high-order-regularization_b200"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(ROOT, "high-order-regularization_b200", "data", "warmstart_h64.hrmlp")


def _data(n=700, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 12)).astype(np.float32) * 1.5 + 0.3
    T = rng.standard_normal((n, 3)).astype(np.float32)
    mean = rng.standard_normal(12).astype(np.float32) * 0.2
    std = (0.5 + rng.random(12)).astype(np.float32)
    return X, T, mean, std


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _net(ctx, mean, std, scale, seed=5):
    m = highreg.MLP(ctx, seed)
    m.set_normalization(mean, std, scale)
    return m


def test_forward_matches_oracle(ctx):
    X, T, mean, std = _data()
    m = _net(ctx, mean, std, 2.5)
    p = m.params()
    raw = torch.zeros((len(X), 3), dtype=torch.float32, device="cuda")
    out = torch.zeros(3 * len(X), dtype=torch.float64, device="cuda")
    base = _dev(np.arange(3 * len(X), dtype=np.float64))
    m.infer(_dev(X), out=out, base=base, raw=raw)
    torch.cuda.synchronize()
    y, _ = mlp_oracle.forward(p.astype(np.float64), X, mean.astype(np.float64), std.astype(np.float64))
    r = raw.cpu().numpy()
    assert np.abs(r - y).max() <= 2e-5 * max(1.0, np.abs(y).max())
    o = out.cpu().numpy() - np.arange(3 * len(X))
    assert np.abs(o - 2.5 * r.ravel()).max() < 1e-5


def test_inference_rotates_the_output_into_each_frame(ctx):
    X, _, mean, std = _data(n=300, seed=6)
    m = _net(ctx, mean, std, 0.7)
    rng = np.random.default_rng(8)
    rot = np.stack([np.linalg.qr(rng.standard_normal((3, 3)))[0] for _ in range(2)])
    raw = torch.zeros((300, 3), dtype=torch.float32, device="cuda")
    m.infer(_dev(X), raw=raw)
    base = _dev(rng.standard_normal(900))
    out = torch.zeros(900, dtype=torch.float64, device="cuda")
    m.infer_frames(_dev(X), out, base, [0, 120, 300], rot)
    torch.cuda.synchronize()
    r = raw.cpu().numpy().astype(np.float64)
    want = np.concatenate([r[:120] @ rot[0], r[120:] @ rot[1]]) * np.float64(np.float32(0.7))
    got = (out - base).cpu().numpy().reshape(-1, 3)
    assert np.abs(got - want).max() < 1e-6 * max(1.0, np.abs(want).max())


def test_gradient_matches_oracle(ctx):
    """FP32 kernels vs the FP64 oracle: relative to the largest gradient entry."""
    X, T, mean, std = _data()
    m = _net(ctx, mean, std, 1.7)
    p = m.params().astype(np.float64)
    loss, g = m.gradient(_dev(X), _dev(T), len(X))
    lo, go = mlp_oracle.loss_and_grad(p, X, T, mean.astype(np.float64), std.astype(np.float64), 1.7)
    assert abs(loss - lo) <= 1e-5 * lo
    scale = np.abs(go).max()
    assert np.abs(g - go).max() <= 1e-4 * scale
    # per-layer relative L2 error
    o = 0
    for shp in mlp_oracle.SHAPES:
        k = int(np.prod(shp))
        a, b = g[o:o + k], go[o:o + k]
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-9
        o += k


def test_adam_step_matches_oracle(ctx):
    X, T, mean, std = _data(n=256, seed=2)
    m = _net(ctx, mean, std, 1.0)
    p0 = m.params().astype(np.float64)
    _, g = m.gradient(_dev(X), _dev(T), len(X))
    m.train_step(_dev(X), _dev(T), len(X), 1e-3, random=False)
    p1 = m.params().astype(np.float64)
    want, _, _ = mlp_oracle.adam_step(p0, g.astype(np.float64), np.zeros_like(p0), np.zeros_like(p0), 1, 1e-3)
    assert np.abs(p1 - want).max() < 1e-6


def test_training_is_deterministic_and_reduces_the_loss(ctx):
    X, T, mean, std = _data(n=4096, seed=4)
    T = (np.tanh(X[:, :3]) * 0.5 + 0.1 * X[:, 3:6]).astype(np.float32)  # a learnable map
    Xd, Td = _dev(X), _dev(T)
    runs = []
    for _ in range(2):
        m = _net(ctx, mean, std, 1.0, seed=11)
        first = m.train_step(Xd, Td, 512, 3e-3, seed=7, want_loss=True)
        for _ in range(300):
            m.train_step(Xd, Td, 512, 3e-3, seed=7)
        last, _ = m.gradient(Xd, Td, 4096)
        runs.append((first, last, m.params()))
    assert runs[0][1] < 0.2 * runs[0][0]
    assert np.array_equal(runs[0][2], runs[1][2])


def test_weights_file_round_trip_and_rejection(ctx, tmp_path):
    X, T, mean, std = _data(n=64)
    m = _net(ctx, mean, std, 3.0)
    path = str(tmp_path / "w.hrmlp")
    m.save(path)
    m2 = highreg.MLP(ctx, 99)
    m2.load(path)
    assert np.array_equal(m.params(), m2.params())
    a = torch.zeros(3 * 64, dtype=torch.float64, device="cuda")
    b = torch.zeros(3 * 64, dtype=torch.float64, device="cuda")
    m.infer(_dev(X), out=a)
    m2.infer(_dev(X), out=b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    raw = bytearray(open(path, "rb").read())
    raw[200] ^= 1
    bad = str(tmp_path / "bad.hrmlp")
    open(bad, "wb").write(bytes(raw))
    with pytest.raises(highreg.HrError) as e:
        m2.load(bad)
    assert e.value.code == highreg.HR_ERR_ARG


def test_garbage_guess_falls_back_to_zero_guess(ctx):
    """A network with a huge output scale gives ||b - A x0|| > ||b||: the solver
    drops the guess and still converges to the zero-guess answer."""
    import warmstart

    prob = warmstart.Problem(warmstart.SEED, 450, 16)
    S = warmstart.Solver(ctx, prob, P=4, N0=300, theta=0.6)
    z = S.run(highreg.HR_FP64, tol=1e-10)
    xz = S.x.clone()
    bad = highreg.MLP(ctx, 3)
    bad.set_normalization(np.zeros(12, np.float32), np.ones(12, np.float32), 1e6)
    w = S.run(highreg.HR_FP64, mlp=bad, tol=1e-10)
    assert w["guess_rejected"] == 1
    assert w["iterations"] == z["iterations"]
    assert float(torch.linalg.norm(S.x - xz) / torch.linalg.norm(xz)) < 1e-12


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="no trained weights committed")
def test_trained_network_improves_the_guess(ctx):
    """Held-out instance (index 460, outside the 448 training instances) at
    h = 1/32. What the trained network gains over the method without it: its
    guess is several times closer to the converged solution than the
    physics-only guess (the imposed rigid motion), the solver accepts it and
    converges to the zero-guess answer. GMRES on this second-kind operator
    converges superlinearly from zero, so a guess of ~1% error does not cut
    the iteration count; the test pins that it costs at most one iteration."""
    import warmstart

    mlp = highreg.MLP(ctx, 0)
    mlp.load(WEIGHTS)
    prob = warmstart.Problem(warmstart.SEED, 460, 32)
    S = warmstart.Solver(ctx, prob, P=6, N0=2000, theta=0.6)
    z = S.run(highreg.HR_FP64, tol=1e-10)
    xz = S.x.clone()
    g = S.guess(mlp)
    err_guess = float(torch.linalg.norm(g - xz) / torch.linalg.norm(xz))
    err_imposed = float(torch.linalg.norm(S.uimp - xz) / torch.linalg.norm(xz))
    w = S.run(highreg.HR_FP64, mlp=mlp, tol=1e-10)
    print("guess error %.3e (imposed motion only %.3e); iterations zero %d learned %d"
          % (err_guess, err_imposed, z["iterations"], w["iterations"]))
    assert w["guess_rejected"] == 0
    assert err_guess < 0.5 * err_imposed
    assert w["iterations"] <= z["iterations"] + 1
    assert float(torch.linalg.norm(S.x - xz) / torch.linalg.norm(xz)) < 1e-8


def test_closing_the_context_closes_its_objects():
    """Plans and networks made on a context are released before it, whatever
    order the caller drops them in."""
    import warmstart

    c = highreg.Context(0)
    prob = warmstart.Problem(warmstart.SEED, 450, 12)
    plan = highreg.Plan2S(c, prob.geo, mode=highreg.HR_TREE, P=4, N0=300, theta=0.6)
    m = highreg.MLP(c, 1)
    c.close()
    assert plan.p is None and m.p is None
    del plan, m
