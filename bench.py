#!/usr/bin/env python
"""Benchmark of the two-surface boundary-integral solve on B200.

Workload (one "step"): the two-surface problem of highreg_stokes_2surf at
h = 1/64 (27,934 + 29,084 quadrature points, n = 171,054 unknowns), KITC
treecode P = 6, N0 = 2000, theta = 0.6: the right-hand side b = -2/3 S[f]
(four Stokeslet sums) and the GMRES solve of (I - 2/3 D) u = b to a 1e-10
relative residual (restart 50), all on the device, FP64.

value: pair interactions per second of the whole step (regularized and plain
target-source pairs plus target-proxy pairs), summed over ranks and divided
by the slowest rank's time. Each timed step is preceded by an L2 flush
(a 256 MB device write) outside its CUDA-event pair.

--impl reference times the reference's own CPU implementation (the
unmodified highreg_stokes_2surf compiled into oracle/_ref) on the host cores:
each step is one reference operator application solve_IE_1step at the same
geometry and treecode parameters; its pairs/s uses the same pair count.

Multi-GPU: the path does not shard (one B200 per problem); --gpus N runs N
independent replicas, one per rank, with no data-path collective.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "high-order-regularization_b200"))

H_INV = 64
P, N0, THETA = 6, 2000, 0.6
INNER = None  # (P, N0) of the inner treecode of the mixed solve's GMRES-IR cycles
RESTART, TOL = 50, 1e-10


def dist_info():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            # raw samples: HR_CLOCKS_DIR if set, else the system temporary directory
            d = os.environ.get("HR_CLOCKS_DIR") or tempfile.gettempdir()
            os.makedirs(d, exist_ok=True)
            self.path = os.path.join(d, "clocks_bench_%d.csv" % self.device)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def pairs_of(work):
    return work["direct_pairs_near"] + work["direct_pairs_far"] + work["proxy_pairs"]


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo; None where unreadable)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference_matvec(geo_pairs, seconds_budget=None):
    """One reference operator application on the host cores (oracle/_ref),
    and, for a kernel-for-kernel figure, the reference's four stresslet
    treecode sums of that operator alone (eval_Stokes_DL_{on,off}Surf_tree,
    without its serial density-interpolation search): returns (R, seconds of
    the operator, seconds of the four sums)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    from oracle import Ref2S

    R = Ref2S(P, N0).setup(H_INV)
    u = np.random.default_rng(0).standard_normal(3 * sum(R.nq))
    t0 = time.perf_counter()
    R.matvec(u)
    dt = time.perf_counter() - t0
    # the matvec left the density and its nearest-point interpolation in the scene
    t0 = time.perf_counter()
    for s, t in ((0, 0), (0, 1), (1, 0), (1, 1)):
        R.eval(1, True, s, t)
    dt_sums = time.perf_counter() - t0
    return R, dt, dt_sums


def run_reference_solve_estimate(args, rank):
    """The reference's CPU solve at h = 1/256 (P = 10, N0 = 8000) estimated
    from its parts, for the GPU solve times the default run reports: the
    reference's right-hand side eval_SL once and its operator application
    solve_IE_1step once (with, alone, its serial interpolate_DL_density and
    its four stresslet treecode sums), timed on the host cores, then
    RHS + iterations x operator with the iteration count of the FP64 solve
    (12 at restart 50). The scene is this library's geometry, which equals the
    reference's own bit for bit; the reference's set-up (its O(Nt Nq)
    nearest-point scan) is not timed. Tens of minutes of host time: not part
    of the default run."""
    if rank != 0:
        return
    import numpy as np

    import highreg

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Ref2S

    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    geo = highreg.Geometry2S(256).scene
    R = Ref2S(10, 8000).load(geo, g=[geo["f0"], geo["f1"]])
    t0 = time.perf_counter()
    R.rhs()
    t_rhs = time.perf_counter() - t0
    u = np.random.default_rng(0).standard_normal(3 * sum(R.nq))
    t0 = time.perf_counter()
    R.matvec(u)
    t_mv = time.perf_counter() - t0
    t0 = time.perf_counter()
    for s in (0, 1):
        R.interpolate(s)
    t_interp = time.perf_counter() - t0
    t0 = time.perf_counter()
    for s, t in ((0, 0), (0, 1), (1, 0), (1, 1)):
        R.eval(1, True, s, t)
    t_sums = time.perf_counter() - t0
    iters = 12
    est = t_rhs + iters * t_mv
    print(json.dumps({"impl": "reference", "workload": "two-surface solve h=1/256 (n=%d), KITC P=10 N0=8000 "
                      "theta=0.6" % (3 * sum(R.nq)), "cores": int(os.environ["OMP_NUM_THREADS"]),
                      "cpu_model": cpu_model(), "seconds_rhs": t_rhs, "seconds_operator": t_mv,
                      "seconds_interpolation": t_interp, "seconds_stresslet_sums": t_sums,
                      "iterations": iters, "solve_seconds_estimated": est,
                      "note": "RHS + 12 operator applications, each part timed once on the host cores"}))


def run_reference(args, rank, world):
    if rank != 0:
        return
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Ref2S, ref_available

    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    line = {"impl": "reference", "metric": "2-surf solve time to 1e-10 residual (plain FP64 vs mixed+warm-start); pairs/s",
            "unit": "pairs/s", "higher_is_better": True, "n_gpus": args.gpus}
    if not ref_available():
        line["unavailable"] = "reference build (oracle/_ref) not present on this machine"
        print(json.dumps(line))
        return
    R = Ref2S(P, N0).setup(H_INV)
    # pair count of one operator application (target-source plus target-proxy
    # evaluations of its four treecode sums), from the oracle's statistics on
    # the reference's own geometry; the count does not depend on the density
    from oracle import Oracle

    orc = Oracle()
    geo = R.geometry()
    n_pairs = 0
    for s, t in [(0, 0), (0, 1), (1, 0), (1, 1)]:
        xq, nrm, area = geo["xq%d" % s], geo["nrm%d" % s], geo["area%d" % s]
        zero = np.zeros(len(xq))
        if s == t:
            _, st = orc.kitc(2, P, N0, THETA, geo["ctr%d" % s], R.DEL, xq, nrm, area, zero)
        else:
            _, st = orc.kitc(3, P, N0, THETA, geo["ctr%d" % s], R.DEL, xq, nrm, area, zero, xt=geo["xq%d" % t],
                             b=geo["b%d" % t], x0=geo["x0%d" % t], n0=geo["n0%d" % t], dens0=np.zeros(len(geo["xq%d" % t])))
        n_pairs += int(st[0] + st[1])
    u = np.random.default_rng(0).standard_normal(3 * sum(R.nq))
    for _ in range(args.warmup):
        R.matvec(u)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        R.matvec(u)
        times.append(time.perf_counter() - t0)
    t = sum(times)
    value = n_pairs * args.steps / t if n_pairs else None
    line.update({"value": value, "steps": args.steps, "warmup": args.warmup,
                 "ms_per_step": 1e3 * t / args.steps, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                 "data": "synthetic (reference geometry generated in-process)",
                 "config": {"workload": "two-surface operator application solve_IE_1step, h=1/64, KITC P=6 N0=2000 theta=0.6",
                            "pairs_per_step": n_pairs},
                 "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                                  "kind": "reference", "cpu_model": cpu_model(),
                                  "sample": "%d reference matvecs (solve_IE_1step) at h=1/64" % args.steps},
                 "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(line))


def warm_guess_fn(ctx, geo, dev):
    """The learned warm start for the bench's scene (the reference's default
    two-spheroid geometry, no imposed motion): returns a function that writes
    the guess into a device vector, and the host time of the features."""
    import numpy as np
    import torch

    import highreg
    import warmstart

    if not os.path.exists(warmstart.DEFAULT_WEIGHTS):
        return None, None
    w = highreg.WarmInstance()
    w.geom = highreg.Geometry2S.default_params()
    for k in range(3):
        w.xmid[k] = 0.5 * (geo["ctr0"][k] + geo["ctr1"][k])
    t0 = time.perf_counter()
    feat, uimp = highreg.warm_features(geo, w)
    feat_s = time.perf_counter() - t0
    rot = highreg.warm_frames(w)
    n0 = len(geo["area0"])
    starts = [0, n0, feat.shape[0]]
    X = torch.from_numpy(feat).to(dev)
    base = torch.from_numpy(uimp).to(dev)
    mlp = highreg.MLP(ctx, 0)
    mlp.load(warmstart.DEFAULT_WEIGHTS)

    def fn(x):
        mlp.infer_frames(X, x, base, starts, rot)

    fn.keep = (X, base, mlp)
    return fn, feat_s


def fp64_true_residual(plan, b, x):
    """||b - A x|| / ||b|| with the plan's FP64 operator (outside any timed region)."""
    import torch

    y = torch.empty_like(x)
    plan.matvec_dev(x, y)
    torch.cuda.synchronize()
    return float(torch.linalg.vector_norm(b - y) / torch.linalg.vector_norm(b))


def timed_solves(plan, stream, flush, f1, f2, b, x, prec, steps, guess=None):
    """steps x (L2 flush; RHS + optional guess + GMRES), CUDA events on the plan's stream."""
    import torch

    times, reps = [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.rhs_dev(f1, f2, b)
        if guess is not None:
            guess(x)
        rep = plan.solve_dev(b, x, use_guess=guess is not None, restart=RESTART, tol=TOL, precision=prec)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        reps.append(rep)
    r = reps[-1]
    # the plain FP64 solve stops on GMRES's recurrence residual; its FP64 true
    # residual is computed here, after the timed steps (the reduced-precision
    # solves compute theirs inside, as their stopping test)
    true_res = r["true_residual"] if r["true_residual"] >= 0.0 else fp64_true_residual(plan, b, x)
    return {"ms_per_step": sum(times) / len(times), "ms_min": min(times), "ms_max": max(times),
            "gmres_iterations": r["iterations"],
            "matvecs_fp64": r["matvecs_fp64"], "matvecs_mixed": r["matvecs_mixed"], "residual": r["residual"],
            "true_residual": true_res, "guess_rejected": r["guess_rejected"]}


def solve_variants(ctx, plan, geo, dev, steps, inner, with_warm=True):
    """The metric's comparison on one plan, each variant after one untimed
    solve (the reduced-precision batches are built on first use): plain FP64,
    mixed precision (GMRES-IR on the plan's treecode), mixed + learned warm
    start and, with an inner treecode (P, N0), mixed and mixed + warm start
    with the inner cycles on it (the FP64 true residuals keep the plan's
    treecode)."""
    import torch

    import highreg

    n = plan.n
    f1 = torch.tensor(geo["f0"], dtype=torch.float64, device=dev)
    f2 = torch.tensor(geo["f1"], dtype=torch.float64, device=dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    stream = torch.cuda.ExternalStream(plan.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    variants = {}
    names = (("fp64", highreg.HR_FP64), ("mixed", highreg.HR_MIXED)) if inner is None else (("fp64", highreg.HR_FP64),)
    for name, pr in names:
        timed_solves(plan, stream, flush, f1, f2, b, x, pr, 1)
        variants[name] = timed_solves(plan, stream, flush, f1, f2, b, x, pr, steps)
    guess, feat_s = warm_guess_fn(ctx, geo, dev) if with_warm else (None, None)
    if guess is not None and inner is None:
        timed_solves(plan, stream, flush, f1, f2, b, x, highreg.HR_MIXED, 1, guess)
        v = timed_solves(plan, stream, flush, f1, f2, b, x, highreg.HR_MIXED, steps, guess)
        v["features_host_ms"] = 1e3 * feat_s
        variants["mixed_warm"] = v
    ms_dl_inner = None
    if inner is not None:
        inner_err = plan.set_inner_tree(inner[0], inner[1], THETA)
        for name, g in (("mixed_inner", None), ("mixed_inner_warm", guess)):
            if name.endswith("warm") and g is None:
                continue
            timed_solves(plan, stream, flush, f1, f2, b, x, highreg.HR_MIXED, 1, g)
            v = timed_solves(plan, stream, flush, f1, f2, b, x, highreg.HR_MIXED, steps, g)
            v["inner_tree"] = {"P": inner[0], "N0": inner[1], "theta": THETA, "rel_l2_error": inner_err}
            if g is not None:
                v["features_host_ms"] = 1e3 * feat_s
            variants[name] = v
        plan.matvec_dev(x, b, highreg.HR_MIXED)
        ms_dl_inner = plan.time_batch(3, 10)
        plan.set_inner_tree(0, 0, THETA)
    for v in variants.values():
        v["speedup_vs_fp64"] = variants["fp64"]["ms_per_step"] / v["ms_per_step"]
    del guess  # releases the network before the context goes
    torch.cuda.synchronize()
    return variants, ms_dl_inner


def run_h256_block(ctx, dev, steps):
    """The precision study's configuration, timed in the same run: the
    two-surface solve at h = 1/256 (n = 2,740,992), KITC P = 10, N0 = 8000,
    GMRES(50) to 1e-10; plain FP64 against mixed precision with the inner
    treecode P = 5, N0 = 2000 (and with the learned warm start)."""
    import highreg

    t0 = time.perf_counter()
    geo = highreg.Geometry2S(256).scene
    plan = highreg.Plan2S(ctx, geo, mode=highreg.HR_TREE, P=10, N0=8000, theta=THETA)
    setup_s = time.perf_counter() - t0
    variants, ms_inner = solve_variants(ctx, plan, geo, dev, steps, (5, 2000))
    out = {"workload": "two-surface solve h=1/256 (n=%d), KITC P=10 N0=8000 theta=0.6, GMRES restart 50 tol 1e-10"
                       % plan.n,
           "steps": steps, "setup_seconds": setup_s, "variants": variants,
           "ms_per_launch_mixed_inner_tree": ms_inner,
           "target": "mixed + learned warm start >= 3x plain FP64"}
    plan.close()
    return out


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    import highreg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    geo = highreg.Geometry2S(H_INV).scene
    ctx = highreg.Context(local_rank)
    plan = highreg.Plan2S(ctx, geo, mode=highreg.HR_TREE, P=P, N0=N0, theta=THETA)
    n = plan.n
    f1 = torch.tensor(geo["f0"], dtype=torch.float64, device=dev)
    f2 = torch.tensor(geo["f1"], dtype=torch.float64, device=dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    prec = highreg.HR_MIXED if args.precision == "mixed" else highreg.HR_FP64
    w_rhs = plan.work(1)
    w_mv = plan.work(0)
    stream = torch.cuda.ExternalStream(plan.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()

    def step():
        plan.rhs_dev(f1, f2, b)
        return plan.solve_dev(b, x, restart=RESTART, tol=TOL, precision=prec)

    for _ in range(max(3, args.warmup)):
        rep = step()
    torch.cuda.synchronize()
    barrier(world)
    clk = ClockSampler(local_rank)
    clk.start()
    l0 = ctx.launches
    times, reps = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        reps.append(rep)
    torch.cuda.synchronize()
    launches = ctx.launches - l0
    clocks = clk.stop()
    barrier(world)

    # the metric's comparison on the same workload and protocol: plain FP64,
    # mixed precision, and mixed precision with the learned warm start
    true_res_main = fp64_true_residual(plan, b, x) if prec == highreg.HR_FP64 else reps[-1]["true_residual"]
    variants, ms_dl_inner = solve_variants(ctx, plan, geo, dev, args.steps, INNER)
    t_local = sum(times) / 1e3
    it = reps[-1]["iterations"]
    mv_per_step = reps[-1]["matvecs_fp64"] + reps[-1]["matvecs_mixed"]
    pairs_step = pairs_of(w_rhs) + mv_per_step * pairs_of(w_mv)
    t_max = max_over_ranks(t_local, world)
    pairs_total = sum_over_ranks(pairs_step * args.steps, world)
    value = pairs_total / t_max

    # dominant kernel: the stresslet batch of the operator (one launch per matvec)
    plan.matvec_dev(x, b)
    ms_dl = plan.time_batch(0, 20)
    ms_dl_mixed = plan.time_batch(2, 20)
    moment_flops = 2.0 * 12 * w_mv["moment_terms"]
    fl_launch = w_mv["flops"] - moment_flops
    peak = ctx.fp64_peak()
    peak32 = ctx.fp32_peak()
    achieved = fl_launch / (ms_dl * 1e-3)
    roofline = {"bound": "fp64", "kernel": "eval_kernel<F_DL> (stresslet batch, one launch per matvec)",
                "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "flops_per_launch": fl_launch, "ms_per_launch": ms_dl,
                "ms_per_launch_mixed_precision": ms_dl_mixed,
                "ms_per_launch_mixed_inner_tree": ms_dl_inner,
                "peak_source": "measured FP64 FMA loop (hr_measure_fp64_peak) on this GPU",
                "peak_fp32": peak32 / 1e12}
    if H_INV == 64 and P == 6 and N0 == 2000:
        # dram__bytes_read.sum + dram__bytes_write.sum of this launch from one ncu capture
        # of both kernels of the batch at this workload: sources are staged once per tile,
        # so DRAM traffic is tiny next to the compute; the bound is the FP64 pipe
        roofline["traffic"] = 10836992 + 157952 + 10935808 + 0
        roofline["traffic_source"] = "ncu capture of this kernel at this workload"

    # end to end through the C ABI with host buffers: scene upload + plan
    # (trees, interaction lists, stencils) + RHS + solve + solution read back
    e2e_times, plan_times, dev_times = [], [], []
    h2d = sum(np.asarray(v).nbytes for k, v in geo.items() if isinstance(v, np.ndarray))
    n_e2e = max(1, min(args.steps, 7 if H_INV <= 64 else 3))
    for k_e2e in range(n_e2e + 1):  # the first pass warms the host-buffer path and is not timed
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p2 = highreg.Plan2S(ctx, geo, mode=highreg.HR_TREE, P=P, N0=N0, theta=THETA)
        t1 = time.perf_counter()
        bh = p2.rhs(geo["f0"], geo["f1"])
        xh, r2 = p2.solve(bh, restart=RESTART, tol=TOL)
        t2 = time.perf_counter()
        p2.close()
        if k_e2e > 0:
            e2e_times.append(t2 - t0)
            plan_times.append(t1 - t0)
            dev_times.append(r2["seconds"])
    e2e_t = max_over_ranks(statistics.median(e2e_times), world)
    e2e = {"value": sum_over_ranks(pairs_step, world) / e2e_t, "unit": "pairs/s", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(8 * n), "seconds_per_step": e2e_t,
           "samples_seconds": [round(t, 4) for t in e2e_times],
           "plan_seconds": statistics.median(plan_times),
           "solve_device_seconds": statistics.median(dev_times),
           "note": "scene upload and plan (trees, interaction lists, stencils on the host) + RHS + solve + "
                   "solution read back, through the C ABI with host buffers"}

    # the precision study's h = 1/256 comparison, timed in the same run
    h256 = None
    if world == 1 and H_INV == 64 and not args.no_h256:
        h256 = run_h256_block(ctx, dev, args.h256_steps)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
                _, dt, dt_sums = cpu_reference_matvec(None)
                cpu = {"value": pairs_of(w_mv) / dt, "unit": "pairs/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                       "kind": "reference", "cpu_model": cpu_model(),
                       "sample": "one reference operator application (solve_IE_1step, h=1/%d, P=%d, N0=%d), %.1f s" % (H_INV, P, N0, dt),
                       # kernel for kernel: the same pairs through the reference's four stresslet
                       # treecode sums alone (its operator also runs a serial nearest-point
                       # interpolation search each call, which the plan here does once)
                       "sums_only": {"value": pairs_of(w_mv) / dt_sums, "unit": "pairs/s", "seconds": dt_sums,
                                     "gpu_batch_pairs_per_s": pairs_of(w_mv) / (ms_dl * 1e-3)}}
            except Exception as e:  # reference build absent
                cpu = {"value": None, "unit": "pairs/s", "cores": 0, "kind": "reference",
                       "sample": "unavailable: %s" % e}
        line = {"metric": "2-surf solve time to 1e-10 residual (plain FP64 vs mixed+warm-start); pairs/s",
                "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": 1e3 * t_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (the reference's two-spheroid geometry generated in-process)",
                "config": {"workload": "two-surface solve h=1/%d (n=%d), KITC P=%d N0=%d theta=0.6, GMRES restart 50 tol 1e-10, %s" % (H_INV, n, P, N0, args.precision),
                           "global_batch": world, "parallelism": "replicas" if world > 1 else "single",
                           "l2": "flushed (256 MB write) before each timed step",
                           "gmres_iterations": it, "matvecs_per_step": mv_per_step,
                           "pairs_per_step": pairs_step, "solve_seconds": t_max / args.steps,
                           "final_residual": reps[-1]["residual"], "true_residual": true_res_main,
                           "precision": args.precision, "work_matvec": w_mv, "work_rhs": w_rhs,
                           "variants": variants, "h256": h256},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
                "gpu_launches": launches}
        print(json.dumps(line))
    plan.close()
    ctx.close()
    return line


def run_e2g(args, rank, world, local_rank):
    """Extend-to-grid workload (translating spheroid, h = 3/N): the four
    boundary sums and the four Poisson extensions on the device, run in FP64,
    mixed precision (FP32 beyond 3 delta) and all-pairs FP32, each with its
    error norms against the FP64 grids and against the exact solution."""
    import numpy as np
    import torch

    import highreg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = highreg.Context(local_rank)
    t0 = time.perf_counter()
    e = highreg.E2G(ctx, args.N)
    setup_s = time.perf_counter() - t0
    info = e.info
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    l0 = ctx.launches
    clk = ClockSampler(local_rank)
    variants = {}
    for name, prec in (("fp64", highreg.HR_FP64), ("mixed", highreg.HR_MIXED), ("fp32", highreg.HR_FP32)):
        for _ in range(max(3, args.warmup)):
            e.run(prec)
        if name == "fp64":
            clk.start()
            l0 = ctx.launches
        reps = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            reps.append(e.run(prec))
        if name == "fp64":
            launches = ctx.launches - l0
            clocks = clk.stop()
            e.snapshot()
        err = e.error_norms()
        v = {k: 1e3 * statistics.mean(r[k] for r in reps) for k in ("seconds_sums", "seconds_poisson", "seconds_total")}
        v = {"ms_sums": v["seconds_sums"], "ms_poisson": v["seconds_poisson"], "ms_total": v["seconds_total"]}
        v.update(err)
        variants[name] = v
    for v in variants.values():
        v["speedup_sums_vs_fp64"] = variants["fp64"]["ms_sums"] / v["ms_sums"]
    pairs = info["pairs"]
    t_sums = max_over_ranks(variants["fp64"]["ms_sums"] * 1e-3, world)
    # end to end through the C ABI: host set-up, sums, Poisson solves, the
    # extended u read back into a page-locked buffer allocated once; one
    # untimed pass warms the host allocators, then the median of three passes
    M3 = (args.N + 1) ** 3
    ub = highreg.pinned_empty(3 * M3)
    e2e_times = []
    for k_e2e in range(4):
        t0 = time.perf_counter()
        e2 = highreg.E2G(ctx, args.N)
        e2.run()
        e2.get(3, out=ub)
        dt_e2e = time.perf_counter() - t0
        e2.close()
        if k_e2e > 0:
            e2e_times.append(dt_e2e)
    e2e_s = statistics.median(e2e_times)
    del ub
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline and args.N <= 96:
            try:
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                from oracle import RefE2G

                os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
                R = RefE2G()
                R.setup(args.N)
                t1 = time.perf_counter()
                R.eval_p_faces()
                R.eval_u_faces()
                dt = time.perf_counter() - t1
                face_pairs = 2 * info["n_face"] * info["nq"]
                cpu = {"value": face_pairs / dt, "unit": "pairs/s", "cores": int(os.environ["OMP_NUM_THREADS"]),
                       "kind": "reference",
                       "sample": "the reference's face sums (stokes_pressure_away, stokes_SL_away) at N=%d, %.1f s"
                                 % (args.N, dt)}
            except Exception as ex:
                cpu = {"value": None, "unit": "pairs/s", "cores": 0, "kind": "reference",
                       "sample": "unavailable: %s" % ex}
        line = {"metric": "extend-to-grid boundary sums; pairs/s", "value": sum_over_ranks(pairs, world) / t_sums,
                "unit": "pairs/s", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
                "ms_per_step": variants["fp64"]["ms_total"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (the reference's translating spheroid generated in-process)",
                "config": {"workload": "extend-to-grid N=%d (h=3/%d): %d quadrature points, %d band + %d face targets, "
                                       "4 sums + 4 DST Poisson solves on %d^3" % (args.N, args.N, info["nq"],
                                                                                  info["n_band"], info["n_face"],
                                                                                  args.N - 1),
                           "pairs_per_step": pairs, "host_setup_seconds": setup_s,
                           "l2": "flushed (256 MB write) before each timed step", "variants": variants},
                "cpu_baseline": cpu,
                "e2e": {"value": pairs / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": int(8 * 3 * M3), "seconds_per_step": e2e_s,
                        "samples_seconds": [round(t, 4) for t in e2e_times],
                        "note": "host set-up (quadrature, band tagging) + sums + Poisson + extended u read back "
                                "into page-locked memory; median of three passes after an untimed one"},
                "clocks": clocks, "gpu_launches": launches}
        print(json.dumps(line))
    e.close()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-h256", action="store_true",
                    help="skip the h = 1/256 FP64 / mixed / warm-start comparison of the default run")
    ap.add_argument("--h256-steps", type=int, default=2, help="timed solves per variant in the h = 1/256 block")
    ap.add_argument("--h", type=int, default=64, help="1/h of the workload (64 is the benchmark)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--P", type=int, default=6, help="treecode degree (6 with h=1/64; 10 with h=1/256)")
    ap.add_argument("--N0", type=int, default=2000, help="treecode leaf size (2000 with h=1/64; 8000 with h=1/256)")
    ap.add_argument("--workload", default="2s", choices=["2s", "e2g"],
                    help="2s: the two-surface solve (the benchmark); e2g: the extend-to-grid pipeline")
    ap.add_argument("--N", type=int, default=96, help="extend-to-grid grid size (96 or 384)")
    ap.add_argument("--reference-h256-estimate", action="store_true",
                    help="with --impl reference: time the reference's RHS and one operator application at "
                         "h = 1/256 on the host cores and print the estimated solve time (tens of minutes)")
    ap.add_argument("--inner", default="auto",
                    help="treecode 'P,N0' of the mixed solve's inner operator; 'auto': 5,2000 when the "
                         "workload's P is above 6, 'none': no inner treecode")
    args = ap.parse_args()
    global H_INV, P, N0, INNER
    H_INV, P, N0 = args.h, args.P, args.N0
    if args.inner == "auto":
        INNER = (5, 2000) if P > 6 else None
    elif args.inner == "none":
        INNER = None
    else:
        INNER = tuple(int(v) for v in args.inner.split(","))
    rank, world, local_rank = dist_info()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference" and args.reference_h256_estimate:
            run_reference_solve_estimate(args, rank)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "e2g":
            run_e2g(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
