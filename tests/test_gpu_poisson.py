"""GPU parity of the extend-to-grid Poisson path (fused DST-I pass kernel:
sine pre-twiddle, shared-memory Stockham FFT, real split and recurrence;
4th-order compact RHS) against the reference's golden outputs
(E2G/main.cpp:969-1044, 1423-1823)."""
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


@pytest.mark.parametrize("n", [1, 3, 5, 13, 21, 47, 95, 127, 191, 193])
def test_dst_poisson_line_lengths(ctx, oracle, n):
    # every FFT stage kind of the shared-memory pass: none (n = 1), radix 2,
    # 3, 4, 8 and direct prime stages (7, 11, 97), and the register pass
    # (n = 64 R - 1: 127 with R = 2, 191 with R = 3), against the oracle's
    # direct O(n^4) transform
    f = np.random.default_rng(n).standard_normal(n ** 3)
    assert rel_err(ctx.dst_poisson3d(n, f), oracle.dst_poisson(n, f)) < 1e-12


@pytest.mark.parametrize("n", [255, 383, 511])
def test_dst1_register_pass_full_lines(ctx, n):
    # the register pass at R = 4, 6 (the N = 384 grid), 8: the plain 3D DST-I
    # against scipy's DST-I (type 1, unnormalised: FFTW's RODFT00) on the
    # whole cube
    import scipy.fft as sf

    f = np.random.default_rng(n).standard_normal(n ** 3)
    got = ctx.dst1_3d(n, f).reshape(n, n, n)
    ref = sf.dstn(f.reshape(n, n, n), type=1, workers=-1)
    assert rel_err(got, ref) < 1e-12


def test_dst_poisson_full_size_operator(ctx):
    # n = 383, the line length of the N = 384 grid: the 4th-order compact
    # operator (2/3)(lap7 + (sum of the 8 corners - 8u)/8) applied to the
    # zero-padded solution returns the data
    n = 383
    f = np.random.default_rng(383).standard_normal(n ** 3)
    U = np.zeros((n + 2,) * 3)
    U[1:-1, 1:-1, 1:-1] = ctx.dst_poisson3d(n, f).reshape(n, n, n)
    c = U[1:-1, 1:-1, 1:-1]
    S = slice(1, -1)
    sh = {-1: slice(0, -2), 0: S, 1: slice(2, None)}
    Lu = -6.0 * c
    for a, b, e in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        Lu += U[sh[a], sh[b], sh[e]]
    Lu -= c
    for a in (-1, 1):
        for b in (-1, 1):
            for e in (-1, 1):
                Lu += U[sh[a], sh[b], sh[e]] / 8.0
    Lu *= 2.0 / 3.0
    assert rel_err(Lu.ravel(), f) < 1e-9


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
