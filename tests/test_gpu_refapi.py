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
    # the written solution against the checker's solve of the same system
    import highreg

    G = highreg.Geometry2S(32).scene
    sc = oracle.scene(G, tree=True, P=6, N0=1000)
    b = oracle.rhs_2s(sc, G["f0"], G["f1"])
    x, _ = oracle.gmres_2s(sc, b, im=15)
    v1 = np.loadtxt(os.path.join(tmp_path, "vel1_N32_highreg_57_k4")).ravel()
    v2 = np.loadtxt(os.path.join(tmp_path, "vel2_N32_highreg_57_k4")).ravel()
    assert rel_err(np.concatenate([v1, v2]), x) < 1e-9
