"""Learned GMRES warm start for the two-surface solve.

Pipeline (every numeric step on the device through libhighreg_b200.so):

1. instances: ``hr_warm_instance_make(seed, i)`` — the reference's spheroid
   pair with a random gap, relative rotation and imposed rigid motion; scene
   set-up by the product's geometry generator (host C++);
2. data: each instance is solved by the method itself (FP64 boundary sums,
   GMRES to 1e-10); a sample is one quadrature point, its 12 features
   (``hr_warm_features``) and its target, the converged solution minus the
   imposed velocity;
3. training: Adam on the mean squared error with the CUDA forward / backward /
   Adam kernels (``hr_mlp_train_step``), batches drawn on the device; targets
   and vector features are in the body frame of the point's own surface;
4. use: ``hr_mlp_infer_frames`` writes guess = u_imposed + R^T MLP(features)
   straight into the solver's device vector; GMRES checks ||b - A x0|| <= ||b||
   and falls back to the zero guess otherwise, so only iterations and time
   change.

Command line::

    python warmstart.py train --out weights.hrmlp --report report.json
    python warmstart.py evaluate --weights weights.hrmlp --report report.json

The committed weights (``data/warmstart_h64.hrmlp``) were made by ``train``
with the defaults below.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import queue
import sys
import threading
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)
import highreg as hr  # noqa: E402

SEED = 20261203
N_INSTANCES = 512
N_TRAIN = 448
DEFAULT_WEIGHTS = os.path.join(HERE, "data", "warmstart_h64.hrmlp")
TREE = dict(P=6, N0=2000, theta=0.6)


class Problem:
    """One seeded instance at h = 1/N: scene, features, imposed velocity."""

    def __init__(self, seed: int, index: int, N: int):
        self.index, self.N = index, N
        self.inst = hr.warm_instance(seed, index)
        t0 = time.perf_counter()
        self.geo = hr.Geometry2S(N, self.inst.geom).scene
        t1 = time.perf_counter()
        self.feat, self.uimp = hr.warm_features(self.geo, self.inst)
        self.rot = hr.warm_frames(self.inst)
        self.t_geometry = t1 - t0
        self.t_features = time.perf_counter() - t1
        self.n0 = len(self.geo["area0"])
        self.n = 3 * (self.n0 + len(self.geo["area1"]))
        self.starts = [0, self.n0, self.n // 3]


def problems(seed: int, indices, N: int, depth: int = 2):
    """Yields Problems, building the next ones on a host thread meanwhile."""
    q: queue.Queue = queue.Queue(maxsize=depth)

    def work():
        try:
            for i in indices:
                q.put(Problem(seed, i, N))
        except BaseException as e:  # surface the error in the consumer
            q.put(e)
        q.put(None)

    th = threading.Thread(target=work, daemon=True)
    th.start()
    while True:
        item = q.get()
        if item is None:
            break
        if isinstance(item, BaseException):
            raise item
        yield item
    th.join()


class Solver:
    """Device-resident two-surface solve of one Problem: b = rhs(f) + 2/3 u_imposed."""

    def __init__(self, ctx: hr.Context, prob: Problem, P=6, N0=2000, theta=0.6):
        self.ctx, self.prob = ctx, prob
        self.plan = hr.Plan2S(ctx, prob.geo, mode=hr.HR_TREE, P=P, N0=N0, theta=theta)
        b = self.plan.rhs(prob.geo["f0"], prob.geo["f1"]) + (2.0 / 3.0) * prob.uimp
        dev = torch.device("cuda", torch.cuda.current_device())
        self.b = torch.from_numpy(b).to(dev)
        self.uimp = torch.from_numpy(prob.uimp).to(dev)
        self.feat = torch.from_numpy(prob.feat).to(dev)
        self.rot = torch.from_numpy(prob.rot).to(dev)
        self.x = torch.zeros_like(self.b)
        torch.cuda.synchronize()
        self.stream = torch.cuda.ExternalStream(self.plan.stream())

    def body_frame(self, v):
        """(n/3, 3) world-frame rows -> body frame of each point's surface."""
        v = v.view(-1, 3)
        n0 = self.prob.n0
        return torch.cat([v[:n0] @ self.rot[0].T, v[n0:] @ self.rot[1].T])

    def run(self, precision=hr.HR_FP64, mlp: hr.MLP | None = None, tol=1e-10, restart=50, max_iter=200,
            features_ms=0.0, guess: str | None = None):
        """Returns the GMRES report with ``ms`` = device time of guess + solve.
        guess: None (zero), "mlp" (needs mlp) or "imposed" (x0 = u_imposed)."""
        if mlp is not None and guess is None:
            guess = "mlp"
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(self.stream)
        if guess == "mlp":
            mlp.infer_frames(self.feat, self.x, self.uimp, self.prob.starts, self.prob.rot)
        elif guess == "imposed":
            with torch.cuda.stream(self.stream):
                self.x.copy_(self.uimp)
        rep = self.plan.solve_dev(self.b, self.x, use_guess=guess is not None, restart=restart, tol=tol,
                                  max_iter=max_iter, precision=precision, check=False)
        e1.record(self.stream)
        e1.synchronize()
        rep["ms"] = e0.elapsed_time(e1)
        rep["ms_with_features"] = rep["ms"] + (features_ms if guess == "mlp" else 0.0)
        rep.pop("resid_hist", None)
        return rep

    def guess(self, mlp: hr.MLP):
        g = torch.empty_like(self.b)
        mlp.infer_frames(self.feat, g, self.uimp, self.prob.starts, self.prob.rot)
        torch.cuda.synchronize()
        return g


def generate(ctx, seed, indices, N, log=print, tol=1e-10):
    """Solves each instance (FP64) and returns device (X, T) plus per-instance records."""
    Xs, Ts, recs = [], [], []
    s1 = np.zeros(hr.NFEAT)
    s2 = np.zeros(hr.NFEAT)
    for prob in problems(seed, indices, N):
        S = Solver(ctx, prob, **TREE)
        rep = S.run(hr.HR_FP64, tol=tol)
        if rep["residual"] > tol:
            raise RuntimeError("instance %d did not converge: %r" % (prob.index, rep))
        Xs.append(S.feat)
        Ts.append(S.body_frame(S.x - S.uimp).float())
        f64 = prob.feat.astype(np.float64)
        s1 += f64.sum(0)
        s2 += (f64 * f64).sum(0)
        recs.append(dict(index=prob.index, n=prob.n, gap=prob.inst.gap, iterations=rep["iterations"],
                         ms=rep["ms"], t_geometry=prob.t_geometry))
        if len(recs) % 32 == 0:
            log("  instance %d: n=%d gap=%.3f iterations=%d %.1f ms" % (prob.index, prob.n, prob.inst.gap,
                                                                       rep["iterations"], rep["ms"]))
        del S
    X = torch.cat(Xs)
    T = torch.cat(Ts)
    npts = X.shape[0]
    mean = s1 / npts
    std = np.sqrt(np.maximum(s2 / npts - mean * mean, 1e-12))
    return X, T, mean, std, recs


def train(ctx, X, T, mean, std, steps=100000, batch=16384, lr0=2e-3, lr1=2e-5, seed=SEED, log=print):
    """Adam with cosine-decayed learning rate; returns (mlp, loss history)."""
    out_scale = float(torch.sqrt((T.double() ** 2).mean()).item())
    mlp = hr.MLP(ctx, seed)
    mlp.set_normalization(mean.astype(np.float32), std.astype(np.float32), out_scale)
    hist = []
    t0 = time.perf_counter()
    for k in range(steps):
        lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + math.cos(math.pi * k / max(1, steps - 1)))
        want = k % 5000 == 0 or k == steps - 1
        loss = mlp.train_step(X, T, batch, lr, seed=seed, random=True, want_loss=want)
        if want:
            hist.append((k, loss))
            log("  step %6d  lr %.2e  loss %.4e" % (k, lr, loss))
    torch.cuda.synchronize()
    return mlp, hist, time.perf_counter() - t0, out_scale


def evaluate(ctx, mlp, seed, indices, N, log=print, tol=1e-10):
    """Zero vs learned guess, FP64 and mixed, on each instance."""
    rows = []
    for prob in problems(seed, indices, N):
        S = Solver(ctx, prob, **TREE)
        feat_ms = prob.t_features * 1e3
        z64 = S.run(hr.HR_FP64, tol=tol)
        xz = S.x.clone()
        g = S.guess(mlp)
        guess_err = float(torch.linalg.norm(g - xz) / torch.linalg.norm(xz))
        base_err = float(torch.linalg.norm(S.uimp - xz) / torch.linalg.norm(xz))
        xf = xz - S.uimp
        mlp_xf_err = float(torch.linalg.norm(g - S.uimp - xf) / torch.linalg.norm(xf))
        w64 = S.run(hr.HR_FP64, mlp=mlp, tol=tol, features_ms=feat_ms)
        sol_diff = float(torch.linalg.norm(S.x - xz) / torch.linalg.norm(xz))
        i64 = S.run(hr.HR_FP64, tol=tol, guess="imposed")
        zmx = S.run(hr.HR_MIXED, tol=tol)
        wmx = S.run(hr.HR_MIXED, mlp=mlp, tol=tol, features_ms=feat_ms)
        rows.append(dict(index=prob.index, N=N, n=prob.n, gap=prob.inst.gap, guess_rel_err=guess_err,
                         imposed_only_rel_err=base_err, mlp_rel_err_on_force_response=mlp_xf_err,
                         warm_vs_zero_solution_rel_diff=sol_diff, features_ms=feat_ms, zero_fp64=z64,
                         warm_fp64=w64, imposed_fp64=i64, zero_mixed=zmx, warm_mixed=wmx))
        log("  instance %d N=%d: guess err %.2e (force response %.2e) | iterations zero %d imposed %d warm %d |"
            " ms zero %.1f warm %.1f warm+mixed %.1f"
            % (prob.index, N, guess_err, mlp_xf_err, z64["iterations"], i64["iterations"], w64["iterations"],
               z64["ms"], w64["ms_with_features"], wmx["ms_with_features"]))
        del S
    return rows


def summarize(rows):
    def mean(key, sub):
        return float(np.mean([r[key][sub] for r in rows]))

    s = dict(instances=len(rows),
             iterations=dict(zero_fp64=mean("zero_fp64", "iterations"), warm_fp64=mean("warm_fp64", "iterations"),
                             imposed_fp64=mean("imposed_fp64", "iterations"),
                             zero_mixed=mean("zero_mixed", "iterations"),
                             warm_mixed=mean("warm_mixed", "iterations")),
             ms=dict(zero_fp64=mean("zero_fp64", "ms"), warm_fp64=mean("warm_fp64", "ms_with_features"),
                     imposed_fp64=mean("imposed_fp64", "ms"),
                     zero_mixed=mean("zero_mixed", "ms"), warm_mixed=mean("warm_mixed", "ms_with_features")),
             guess_rel_err=float(np.mean([r["guess_rel_err"] for r in rows])),
             mlp_rel_err_on_force_response=float(np.mean([r["mlp_rel_err_on_force_response"] for r in rows])),
             imposed_only_rel_err=float(np.mean([r["imposed_only_rel_err"] for r in rows])),
             max_solution_rel_diff=float(np.max([r["warm_vs_zero_solution_rel_diff"] for r in rows])),
             guesses_rejected=int(sum(r["warm_fp64"]["guess_rejected"] for r in rows)))
    s["speedup_warm_mixed_vs_zero_fp64"] = s["ms"]["zero_fp64"] / s["ms"]["warm_mixed"]
    s["speedup_warm_fp64_vs_zero_fp64"] = s["ms"]["zero_fp64"] / s["ms"]["warm_fp64"]
    return s


def _range(text):
    a, b = text.split("-")
    return list(range(int(a), int(b) + 1))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", required=True)
    t.add_argument("--report", default=None)
    t.add_argument("--N", type=int, default=64)
    t.add_argument("--instances", type=int, default=N_INSTANCES)
    t.add_argument("--train", type=int, default=N_TRAIN)
    t.add_argument("--steps", type=int, default=100000)
    t.add_argument("--batch", type=int, default=16384)
    t.add_argument("--seed", type=int, default=SEED)
    t.add_argument("--eval-N", type=int, nargs="*", default=[128])
    e = sub.add_parser("evaluate")
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--report", default=None)
    e.add_argument("--N", type=int, default=64)
    e.add_argument("--indices", type=_range, default=_range("448-511"))
    e.add_argument("--seed", type=int, default=SEED)
    e.add_argument("--eval-N", type=int, nargs="*", default=[128])
    a = ap.parse_args(argv)

    log = lambda s: print(s, flush=True)  # noqa: E731
    ctx = hr.Context(0)
    report = dict(seed=a.seed, N=a.N, tree=TREE, tol=1e-10, restart=50)
    if a.cmd == "train":
        t0 = time.perf_counter()
        log("generating %d instances at h=1/%d" % (a.instances, a.N))
        X, T, mean, std, recs = generate(ctx, a.seed, range(a.train), a.N, log)
        report["data"] = dict(instances=a.train, samples=int(X.shape[0]), seconds=time.perf_counter() - t0,
                              mean_iterations=float(np.mean([r["iterations"] for r in recs])),
                              mean_solve_ms=float(np.mean([r["ms"] for r in recs])))
        log("training on %d samples" % X.shape[0])
        mlp, hist, secs, out_scale = train(ctx, X, T, mean, std, steps=a.steps, batch=a.batch, seed=a.seed,
                                           log=log)
        report["training"] = dict(steps=a.steps, batch=a.batch, seconds=secs, loss=hist, out_scale=out_scale)
        mlp.save(a.out)
        del X, T
        held = list(range(a.train, a.instances))
    else:
        mlp = hr.MLP(ctx, 0)
        mlp.load(a.weights)
        held = a.indices
    log("evaluating %d held-out instances at h=1/%d" % (len(held), a.N))
    rows = evaluate(ctx, mlp, a.seed, held, a.N, log)
    report["held_out"] = summarize(rows)
    report["held_out_rows"] = rows
    for N2 in a.eval_N:
        r2 = evaluate(ctx, mlp, a.seed, held[:1], N2, log)
        report["h_1_%d" % N2] = r2[0]
    log(json.dumps(report["held_out"], indent=1))
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(report, fh, indent=1)


if __name__ == "__main__":
    main()
