"""The C++ drop-in layer: the reference's own unmodified two-surface driver
(highreg_stokes_2surf main.cpp, surface.cpp, utilities.cpp) relinked against
libhighreg_refapi.so instead of its treecode and direct-sum sources, so that
every boundary sum of its GMRES solve runs on the B200. Its printed residual
history and written solution must be the reference's (h = 1/32: 13
iterations to 7.8214e-11)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_err

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "ref2s_main_relinked")


@pytest.mark.skipif(not os.path.exists(EXE), reason="relinked reference driver not built")
def test_reference_driver_on_gpu(tmp_path, oracle):
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
    r = subprocess.run([EXE], cwd=tmp_path, capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    m = re.search(r"GMRES converged in (\d+) iterations with residual = ([0-9.eE+-]+)", r.stdout)
    assert m, r.stdout[-2000:]
    assert int(m.group(1)) == 13
    assert abs(float(m.group(2)) - 7.8214e-11) / 7.8214e-11 < 1e-3
    hist = [float(x) for x in re.findall(r"Iteration \d+\s+residual = ([0-9.eE+-]+)", r.stdout)]
    ref_hist = [6.19915e-02, 7.14192e-03, 8.84480e-04, 1.22093e-04, 2.40454e-05, 3.99025e-06, 6.06091e-07,
                1.00332e-07, 2.29270e-08, 6.67164e-09, 1.58622e-09, 3.25818e-10, 7.82140e-11]
    assert np.allclose(hist, ref_hist, rtol=1e-4)
    # the written solution against the oracle's solve of the same system
    import highreg

    G = highreg.Geometry2S(32).scene
    sc = oracle.scene(G, tree=True, P=6, N0=1000)
    b = oracle.rhs_2s(sc, G["f0"], G["f1"])
    x, _ = oracle.gmres_2s(sc, b, im=15)
    v1 = np.loadtxt(os.path.join(tmp_path, "vel1_N32_highreg_57_k4")).ravel()
    v2 = np.loadtxt(os.path.join(tmp_path, "vel2_N32_highreg_57_k4")).ravel()
    assert rel_err(np.concatenate([v1, v2]), x) < 1e-9


E2G_EXE = os.path.join(ROOT, "oracle", "_ref", "refe2g_main_relinked")


def _error_lines(text):
    """(line text without numbers, numbers) of every printed error line."""
    num = r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?"
    out = []
    for line in text.splitlines():
        if "err" in line and "time" not in line.lower():
            out.append((re.sub(num, "#", line).strip(), [float(v) for v in re.findall(num, line)]))
    return out


@pytest.mark.skipif(not os.path.exists(E2G_EXE), reason="relinked reference extend-to-grid driver not built")
def test_reference_e2g_driver_with_gpu_poisson(tmp_path):
    """The reference's unmodified extend-to-grid driver (N = 96, its own CPU
    boundary sums) relinked against the FFTW-API layer, so that every DST-I
    of its four Poisson solves runs on the B200: its printed error tables
    equal those of the same driver on the CPU DST-I stand-in (the reference
    built with oracle/fftw_standin), among them the reference's table
    (u in the band: max 4.2629e-04; u on the grid: max 4.34278e-04; p on the
    grid: max 2.9393e-03). Lines that print times are not compared."""
    import oracle as om

    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()))
    r = subprocess.run([E2G_EXE], cwd=tmp_path, capture_output=True, text=True, timeout=900, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "B200 layer" not in r.stderr, r.stderr[-2000:]
    got = _error_lines(r.stdout)
    R = om.RefE2G().setup(96)
    ref = _error_lines(R.run())
    assert len(got) == len(ref) and len(got) >= 6
    for (lg, vg), (lr, vr) in zip(got, ref):
        assert lg == lr
        assert np.allclose(vg, vr, rtol=2e-5, atol=0), (lg, vg, vr)
    text = r.stdout
    assert "max err (u) = 0.000434278" in text and "max err (p) = 0.0029393" in text, text[-3000:]
