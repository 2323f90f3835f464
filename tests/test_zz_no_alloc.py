"""The allocation-free Stokeslet sum entry point, through the C ABI.

It is meant for callers that cannot call cudaMalloc (a framework allocator
owns the device memory, or the path must not synchronize the device): its
only scratch is a fixed static device array. Checked against the allocating
entry point hr_e2g_stokeslet_away on two calls in a row (the second call
reuses the scratch the first one left behind), within the sum tests' FP64
tolerance. This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import highreg
from conftest import rel_err
import e2g_util

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(xs, area, f, xt):
    L = highreg.lib()
    dev = torch.device("cuda", 0)
    txs = torch.tensor(xs, dtype=torch.float64, device=dev)
    ta = torch.tensor(area, dtype=torch.float64, device=dev)
    tf = torch.tensor(f, dtype=torch.float64, device=dev)
    tt = torch.tensor(xt, dtype=torch.float64, device=dev)
    out = torch.full((len(xt),), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.hr_stokeslet_away_noalloc(p(txs), p(ta), p(tf), len(area), p(tt), len(xt) // 3, p(out),
                                     ctypes.c_void_p(stream.cuda_stream))
    stream.synchronize()
    assert rc == highreg.HR_OK
    return out.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(ctx, ge2g):
    N, h = int(ge2g["N"]), float(ge2g["h"])
    xq, area, f = ge2g["xq"], ge2g["area"], ge2g["f"]
    xt, _ = e2g_util.face_targets(N, h)
    ref = ctx.e2g_sl_away(xq, area, f, xt)
    first = _noalloc(xq, area, f, xt)
    assert rel_err(first, ref) < TOL
    # second call: different targets and density, same shared scratch
    rng = np.random.default_rng(9)
    f2 = rng.standard_normal(len(f))
    xt2 = xt[: 3 * 5001] * 1.01 + 0.003
    ref2 = ctx.e2g_sl_away(xq, area, f2, xt2)
    second = _noalloc(xq, area, f2, xt2)
    assert rel_err(second, ref2) < TOL


def test_noalloc_edge_sizes(ctx):
    # no sources: one empty chunk, every target gets zeros
    rng = np.random.default_rng(21)
    xt = rng.uniform(-2.0, 2.0, 3 * 1000)
    z = _noalloc(np.zeros(0), np.zeros(0), np.zeros(0), xt)
    assert np.array_equal(z, np.zeros(len(xt)))
    # targets near the scratch limit: the source chunks drop from ten to one
    # (and to two at half the limit), so each target sums its sources in fewer,
    # longer runs; checked against the allocating entry point
    nq = 20000
    xs = rng.uniform(-1.0, 1.0, 3 * nq)
    area = rng.uniform(0.5, 1.5, nq) * 1e-4
    f = rng.standard_normal(3 * nq)
    L = highreg.lib()
    L.hr_stokeslet_away_noalloc_max_targets.restype = ctypes.c_longlong
    limit = int(L.hr_stokeslet_away_noalloc_max_targets())
    for nt in (limit, limit // 2 + 1):
        xt = rng.uniform(1.5, 3.0, 3 * nt)
        got = _noalloc(xs, area, f, xt)
        ref = ctx.e2g_sl_away(xs, area, f, xt)
        assert rel_err(got, ref) < TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = highreg.lib()
    L.hr_stokeslet_away_noalloc_max_targets.restype = ctypes.c_longlong
    limit = L.hr_stokeslet_away_noalloc_max_targets()
    assert limit > 1_000_000
    dummy = torch.zeros(3, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = L.hr_stokeslet_away_noalloc(p, p, p, 1, p, ctypes.c_int(int(limit) + 1), p, None)
    assert rc == highreg.HR_ERR_ARG
