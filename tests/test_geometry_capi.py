"""CPU tests of the product library: the host geometry setup against the
reference's own scene, and the C ABI surface (symbols, argument errors)."""
import ctypes
import os
import re

import numpy as np
import pytest

import highreg
from conftest import ROOT


def test_geometry_matches_reference_bitwise(g2s):
    G = highreg.Geometry2S(int(g2s["N"])).scene
    for key in ["xq", "nrm", "area", "plane", "f", "b", "x0", "n0", "f0", "nrst", "i123", "ctr"]:
        for s in (0, 1):
            k = "%s%d" % (key, s)
            assert np.array_equal(np.asarray(G[k]), np.asarray(g2s[k])), k
    assert G["h"] == float(g2s["h"]) and G["DEL"] == float(g2s["DEL"])


def test_geometry_h32_counts():
    # golden counts of the reference at h = 1/32 (N1, N2)
    G = highreg.Geometry2S(32).scene
    assert len(G["area0"]) == 6958 and len(G["area1"]) == 7252
    assert abs(G["DEL"] - 0.10254191950095476) < 1e-15


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref2s_P6_N1000.so")),
                    reason="reference build not present")
def test_geometry_matches_reference_h32():
    from oracle import Ref2S

    ref = Ref2S(6, 1000).setup(32).geometry()
    G = highreg.Geometry2S(32).scene
    for k in ref:
        assert np.array_equal(np.asarray(G[k]), np.asarray(ref[k])), k


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "highreg_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hr_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = highreg.lib()
    names = _header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_refapi_library_exports_reference_signatures():
    import subprocess

    lib = os.path.join(ROOT, "high-order-regularization_b200", "libhighreg_refapi.so")
    out = subprocess.run(["nm", "-DC", lib], capture_output=True, text=True).stdout
    txt = open(os.path.join(ROOT, "include", "highreg_refapi.h")).read()
    names = sorted(set(re.findall(r"\b(eval_Stokes_[A-Za-z_]+|hr_refapi_[a-z_]+)\s*\(", txt)))
    assert len(names) == 11
    for n in names:
        assert re.search(r" T " + n + r"\b", out), n


def test_context_argument_errors():
    L = highreg.lib()
    assert L.hr_ctx_create(0, None) == highreg.HR_ERR_ARG
    assert L.hr_stokes_sl_onsurf(None, None, ctypes.c_double(1.0), None, None, None) == highreg.HR_ERR_ARG
    assert L.hr_plan2s_matvec(None, None, None) == highreg.HR_ERR_ARG


def test_context_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(highreg.HrError) as e:
        highreg.Context(0)
    assert e.value.code == highreg.HR_ERR_NO_DEVICE


def test_geometry_rejects_bad_arguments():
    L = highreg.lib()
    p = highreg.Geometry2S.default_params()
    out = ctypes.c_void_p()
    assert L.hr_geom2s_generate(ctypes.byref(p), 1, ctypes.byref(out)) == highreg.HR_ERR_ARG
    assert L.hr_geom2s_generate(None, 16, ctypes.byref(out)) == highreg.HR_ERR_ARG


def test_fftw_layer_exports_its_header():
    """libhighreg_fftw.so exports every function include/fftw_shim/fftw3.h
    declares, with C linkage (FFTW's names, so a driver links it in place of
    -lfftw3); loading it needs no GPU."""
    import ctypes

    path = os.path.join(ROOT, "high-order-regularization_b200", "libhighreg_fftw.so")
    L = ctypes.CDLL(path)
    txt = open(os.path.join(ROOT, "include", "fftw_shim", "fftw3.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = sorted(set(re.findall(r"\b(fftw_[a-z0-9_]+)\s*\(", txt)))
    assert names == ["fftw_cleanup", "fftw_destroy_plan", "fftw_execute", "fftw_free", "fftw_malloc",
                     "fftw_plan_r2r_3d"]
    for n in names:
        assert hasattr(L, n), n
    # unsupported plans are refused before any device work
    L.fftw_plan_r2r_3d.restype = ctypes.c_void_p
    buf = (ctypes.c_double * 64)()
    assert L.fftw_plan_r2r_3d(4, 4, 4, buf, buf, 7, 7, 7, 64) is None      # n + 1 odd
    assert L.fftw_plan_r2r_3d(3, 3, 5, buf, buf, 7, 7, 7, 64) is None      # not a cube
    assert L.fftw_plan_r2r_3d(3, 3, 3, buf, buf, 3, 7, 7, 64) is None      # not RODFT00
