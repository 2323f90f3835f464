"""GPU parity of the extend-to-grid Poisson path (DST-I via cuFFT with
pre/post-twiddle kernels, 4th-order compact RHS) against the reference's
golden outputs (E2G/main.cpp:969-1044, 1423-1823)."""
import numpy as np
import pytest

from conftest import rel_err
import e2g_util

pytestmark = pytest.mark.gpu


def test_dst_poisson_matches_reference(ctx, ge2g):
    n = int(ge2g["N"]) - 1
    out = ctx.dst_poisson3d(n, ge2g["dst_in"])
    assert rel_err(out, ge2g["dst_out"]) < 1e-12


def test_dst_poisson_round_trip(ctx, oracle):
    # the discrete Laplacian applied to the solution returns the data
    n = 23
    f = np.random.default_rng(5).standard_normal(n ** 3)
    assert rel_err(ctx.dst_poisson3d(n, f), oracle.dst_poisson(n, f)) < 1e-12


def test_solve_poisson_matches_reference(ctx, ge2g):
    N, h = int(ge2g["N"]), float(ge2g["h"])
    b2, out = e2g_util.masks(N, h, ge2g["nrst"], ge2g["band2"])
    p_ext = ctx.solve_poisson(N, 3.0, b2, out, None, ge2g["p_band"], 0)
    assert rel_err(p_ext, ge2g["p_ext"]) < 1e-11
    M = N + 1
    ub = ge2g["u_band"].reshape(3, M ** 3)
    ue = ge2g["u_ext"].reshape(3, M ** 3)
    for v in range(3):
        uu = ctx.solve_poisson(N, 3.0, b2, out, ge2g["p_ext"], ub[v], v + 1)
        assert rel_err(uu, ue[v]) < 1e-11
