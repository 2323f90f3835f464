"""The extend-to-grid pipeline on the device (E2G/main.cpp:107-424): setup and
tagging against the reference's own scene, sums and Poisson extensions
against its golden grids, and the error against the exact translating-body
solution at the reference's default grid (h = 1/32, N = 96)."""
import numpy as np
import pytest

import highreg
from conftest import rel_err
import e2g_util

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def e48(ctx):
    e = highreg.E2G(ctx, 48)
    yield e
    e.close()


def test_setup_matches_reference(e48, ge2g):
    s = e48.scene()
    for k in ("xq", "nrm", "area", "f"):
        assert np.array_equal(s[k], ge2g[k]), k
    assert np.array_equal(s["nrst"], ge2g["nrst"])
    assert np.array_equal(s["band2"], ge2g["band2"])
    assert np.max(np.abs(s["b"] - ge2g["b"])) < 1e-14
    assert np.max(np.abs(s["x0"] - ge2g["x0"])) < 1e-14


def test_pipeline_matches_reference(e48, ge2g):
    e48.run()
    M3 = 49 ** 3
    assert rel_err(e48.get(0), ge2g["p_band"]) < 1e-12
    assert rel_err(e48.get(1), ge2g["u_band"]) < 1e-12
    assert rel_err(e48.get(2), ge2g["p_ext"]) < 1e-11
    assert rel_err(e48.get(3), ge2g["u_ext"]) < 1e-11
    # mixed precision: face sums in FP32, band sums split at r = 3 delta
    e48.run(highreg.HR_MIXED)
    assert rel_err(e48.get(3), ge2g["u_ext"]) < 1e-6
    # every pair in FP32
    e48.run(highreg.HR_FP32)
    e32 = rel_err(e48.get(3), ge2g["u_ext"])
    print("E2G N=48 extended velocity, FP32 pairs vs the reference:", e32)
    assert e32 < 1e-3


def test_read_back_into_page_locked_buffer(e48):
    # the same grids through a caller's page-locked buffer, filled in place
    e48.run()
    ref = e48.get(3)
    buf = highreg.pinned_empty(ref.size)
    buf[:] = np.nan
    got = e48.get(3, out=buf)
    assert got is buf and np.array_equal(got, ref)
    assert np.array_equal(e48.get(2, out=highreg.pinned_empty(ref.size // 3)), e48.get(2))
    with pytest.raises(highreg.HrError):
        e48.get(3, out=highreg.pinned_empty(ref.size - 1))


def _exact_grids(N, h):
    M = N + 1
    p = np.zeros(M ** 3)
    u = np.zeros((3, M ** 3))
    outside = np.zeros(M ** 3, bool)
    for i in range(M):
        for j in range(M):
            for k in range(M):
                g = (i * M + j) * M + k
                levl = e2g_util.phi(i * h, j * h, k * h)
                if levl > 0 or abs(levl) < 1e-12:
                    pe, ue = highreg.e2g_exact(i * h, j * h, k * h)
                    p[g] = pe
                    u[:, g] = ue
                    outside[g] = True
                else:
                    u[0, g] = 1.0
    return p, u, outside


def test_exact_solution_error_table_h32(ctx):
    """E2G N = 96: the reference's own error table (its printed golden values)."""
    e = highreg.E2G(ctx, 96)
    with pytest.raises(highreg.HrError):  # no slices before a run
        e.midplane()
    info = e.info
    assert info["nq"] == 6958 and info["n_tagged"] == 44582 and info["n_band"] == 26810 and info["n_face"] == 55298
    e.run()
    N, h = 96, 3.0 / 96
    M3 = 97 ** 3
    pex, uex, outside = _exact_grids(N, h)
    p = e.get(2)
    u = e.get(3).reshape(3, M3)
    perr = np.abs(p - pex)
    uerr = np.sqrt(np.sum((u - uex) ** 2, axis=0))
    # whole grid (E2G/main.cpp:236-259, 470-497)
    assert abs(perr.max() - 2.9393e-03) / 2.9393e-03 < 1e-3
    assert abs(np.sqrt(np.mean(perr ** 2)) - 1.65368e-05) / 1.65368e-05 < 1e-3
    assert abs(uerr.max() - 4.34278e-04) / 4.34278e-04 < 1e-3
    assert abs(np.sqrt(np.mean(uerr ** 2)) - 1.12517e-05) / 1.12517e-05 < 1e-3
    # band velocity before the extension (E2G/main.cpp:1359-1405)
    ub = e.get(1).reshape(3, M3)
    s = e.scene()
    xs, bs, x0s, n0s, f0s, gb = e2g_util.band_targets(N, h, s["nrst"], s["b"], s["x0"], s["n0"])
    be = np.sqrt(np.sum((ub[:, gb] - uex[:, gb]) ** 2, axis=0))
    assert abs(be.max() - 4.2629e-04) / 4.2629e-04 < 1e-3
    assert abs(np.sqrt(np.mean(be ** 2)) - 2.42985e-05) / 2.42985e-05 < 1e-3
    # the device error norms give the same table
    d = e.error_norms()
    assert abs(d["p_max"] - perr.max()) <= 1e-12 * perr.max()
    assert abs(d["p_rms"] - np.sqrt(np.mean(perr ** 2))) <= 1e-9 * d["p_rms"]
    assert abs(d["u_max"] - uerr.max()) <= 1e-12 * uerr.max()
    assert abs(d["u_rms"] - np.sqrt(np.mean(uerr ** 2))) <= 1e-9 * d["u_rms"]
    assert abs(d["band_u_max"] - be.max()) <= 1e-12 * be.max()
    assert abs(d["band_u_rms"] - np.sqrt(np.mean(be ** 2))) <= 1e-9 * d["band_u_rms"]
    assert d["ref_u_rel_l2"] == -1.0
    # mid-plane y = 1.5 slices gathered on the device (the reference's slice files)
    M, jm = N + 1, N // 2
    sl = e.midplane()
    out_mid = outside.reshape(M, M, M)[:, jm, :]
    assert np.array_equal(sl[0], p.reshape(M, M, M)[:, jm, :])
    # the device and host exact solutions differ by rounding (~1e-16 of |p|, |u| = O(1)),
    # which the error slices see as an absolute difference
    for q, ref in ((1, perr), (2, uerr), (3, pex)):
        want = np.where(out_mid, ref.reshape(M, M, M)[:, jm, :], 0.0)
        assert np.allclose(sl[q], want, rtol=1e-12, atol=1e-13), q
    # precision variants against the FP64 grids and the exact solution
    e.snapshot()
    for prec, tol in ((highreg.HR_MIXED, 1e-7), (highreg.HR_FP32, 1e-3)):
        e.run(prec)
        d2 = e.error_norms()
        print("E2G N=96 precision", prec, d2)
        assert d2["ref_u_rel_l2"] < tol and d2["ref_p_rel_l2"] < tol
        assert abs(d2["u_max"] - d["u_max"]) <= 0.05 * d["u_max"]
    e.close()
