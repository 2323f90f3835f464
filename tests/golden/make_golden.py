"""Generates the golden fixtures of tests/golden/ from the reference itself.

The reference (highreg_stokes_2surf, highreg_stokes_extend_to_grid) is
compiled unmodified into oracle/_ref by oracle/build_oracle.py; this script
drives it through oracle/oracle.py on small cases and stores inputs and
outputs as compressed .npz files. It needs the reference build, so it runs
where the reference tree is available; the fixtures it writes are committed.

  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import build_oracle  # noqa: E402
from oracle import Ref2S, RefE2G  # noqa: E402

SEED = 20261203


def make_2s(N=16, P=4, N0=300):
    R = Ref2S(P, N0).setup(N)
    geo = R.geometry()
    rng = np.random.default_rng(SEED)
    out = {k: np.asarray(v) for k, v in geo.items()}
    out["P"], out["N0"], out["N"] = P, N0, N
    # Stokeslet sums of the interfacial force, tree and direct
    for tree in (0, 1):
        for s, t in [(0, 0), (0, 1), (1, 0), (1, 1)]:
            out["sl_t%d_%d%d" % (tree, s, t)] = R.eval(0, tree, s, t)
    # stresslet sums of a seeded random density
    g = [rng.standard_normal(3 * R.nq[0]), rng.standard_normal(3 * R.nq[1])]
    out["g0"], out["g1"] = g
    R.set_g(0, g[0])
    R.set_g(1, g[1])
    R.interpolate(0)
    R.interpolate(1)
    out["g0interp0"] = R.targets(0)["g0"]
    out["g0interp1"] = R.targets(1)["g0"]
    for tree in (0, 1):
        for s, t in [(0, 0), (0, 1), (1, 0), (1, 1)]:
            out["dl_t%d_%d%d" % (tree, s, t)] = R.eval(1, tree, s, t)
    u = np.concatenate(g)
    out["mv_u"] = u
    out["mv_y"] = R.matvec(u)
    out["rhs"] = R.rhs()
    x, hist = R.solve()
    out["sol_x"] = x
    out["sol_hist"] = hist
    np.savez_compressed(os.path.join(HERE, "ref2s_N%d_P%d_N0%d.npz" % (N, P, N0)), **out)


def make_2s_bench(N=64, P=6, N0=2000, n_sample=4096):
    """The benchmark's two-surface configuration (h = 1/64, KITC P = 6,
    N0 = 2000): the reference's GMRES residual history and, at a seeded sample
    of unknowns, its solution, right-hand side and one operator application
    (of a seeded density). Only samples are stored: the full vectors are
    171,054 doubles each."""
    R = Ref2S(P, N0).setup(N)
    n = 3 * sum(R.nq)
    rng = np.random.default_rng(SEED)
    idx = np.sort(rng.choice(n, n_sample, replace=False)).astype(np.int32)
    u = np.random.default_rng(SEED + 1).standard_normal(n)
    out = dict(N=N, P=P, N0=N0, n=n, idx=idx, mv_seed=SEED + 1)
    out["rhs"] = R.rhs()[idx]
    out["mv_y"] = R.matvec(u)[idx]
    x, hist = R.solve()
    out["sol_x"] = x[idx]
    out["sol_hist"] = hist
    np.savez_compressed(os.path.join(HERE, "ref2s_N%d_P%d_N0%d_sampled.npz" % (N, P, N0)), **out)


def make_e2g(N=48):
    R = RefE2G().setup(N)
    S = R.surface()
    T = R.targets()
    nrst = R.nrst()
    out = dict(N=N, h=R.h, DEL=R.DEL, xq=S["xq"], nrm=S["nrm"], area=S["area"], f=S["f"], b=T["b"],
               x0=T["x0"], n0=T["n0"], band2=T["band2"], nrst=nrst)
    p = R.eval_p_faces()
    out["p_faces"] = p
    p = R.eval_p_band(p)
    out["p_band"] = p
    u = R.eval_u_faces()
    out["u_faces"] = np.concatenate(u)
    u = R.eval_u_band(u)
    out["u_band"] = np.concatenate(u)
    p_ext = R.solve_poisson(0, p, p)
    out["p_ext"] = p_ext
    us = [R.solve_poisson(v + 1, p_ext, u[v]) for v in range(3)]
    out["u_ext"] = np.concatenate(us)
    rng = np.random.default_rng(SEED)
    n = N - 1
    f = rng.standard_normal(n ** 3)
    out["dst_in"] = f
    out["dst_out"] = R.dst_poisson(n, f)
    np.savez_compressed(os.path.join(HERE, "refe2g_N%d.npz" % N), **out)


if __name__ == "__main__":
    built = build_oracle.build_reference()
    if not built:
        sys.exit("reference tree not available; fixtures not regenerated")
    make_2s()
    make_e2g()
    make_2s_bench()
    print(sorted(os.listdir(HERE)))
