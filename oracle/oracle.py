"""ctypes front end of the oracle (test infrastructure only).

``Oracle`` wraps ``oracle/liboracle.so`` (the C restatement of the reference's
hot path); ``Ref2S`` and ``RefE2G`` wrap the reference programs compiled from
their own sources into ``oracle/_ref/`` (present wherever they were built).
Only tests/, the smoke test and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _i(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def _u8(a):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """The plain-C restatement (oracle/highreg_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            import build_oracle  # noqa: local module

            build_oracle.build_oracle_lib()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.or_dl_7ord_onsurf.restype = ctypes.c_double
        L.or_lapl_dl_7ord.restype = ctypes.c_double
        L.or_e2g_p_away_one.restype = ctypes.c_double
        L.or_kitc_eval.restype = ctypes.c_int
        L.or_gmres_2s.restype = ctypes.c_int
        for name in ["or_dl_7ord_onsurf", "or_lapl_dl_7ord"]:
            getattr(L, name).argtypes = [ctypes.c_double, ctypes.c_double] + (
                [_D] if name == "or_lapl_dl_7ord" else [])
        L.or_reg_coeff.argtypes = [ctypes.c_double, _D]
        L.or_sl_7ord.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D]
        L.or_dl_7ord.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D]
        L.or_sl_7ord_onsurf.argtypes = [ctypes.c_double, ctypes.c_double, _D]

    # scalar kernels -------------------------------------------------------
    def reg_coeff(self, lam):
        c = np.zeros(3)
        self.lib.or_reg_coeff(float(lam), _d(c))
        return c

    def sl_7ord(self, r, d, c):
        s = np.zeros(2)
        self.lib.or_sl_7ord(float(r), float(d), _d(_f64(c)), _d(s))
        return s

    def dl_7ord(self, r, d, c):
        s = np.zeros(2)
        self.lib.or_dl_7ord(float(r), float(d), _d(_f64(c)), _d(s))
        return s

    def sl_7ord_onsurf(self, r, d):
        s = np.zeros(2)
        self.lib.or_sl_7ord_onsurf(float(r), float(d), _d(s))
        return s

    def dl_7ord_onsurf(self, r, d):
        return self.lib.or_dl_7ord_onsurf(float(r), float(d))

    def lapl_dl_7ord(self, r, d, c):
        return self.lib.or_lapl_dl_7ord(float(r), float(d), _d(_f64(c)))

    # direct sums ----------------------------------------------------------
    def sl_offsurf_direct(self, DEL, xq, nrm, area, f, xt, b, f0, n0):
        nt = len(b)
        out = np.zeros(3 * nt)
        self.lib.or_sl_offsurf_direct(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                                      _d(_f64(area)), _d(_f64(f)), nt, _d(_f64(xt)), _d(_f64(b)),
                                      _d(_f64(f0)), _d(_f64(n0)), _d(out))
        return out

    def sl_onsurf_direct(self, DEL, xq, nrm, area, f):
        out = np.zeros(3 * len(area))
        self.lib.or_sl_onsurf_direct(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                                     _d(_f64(area)), _d(_f64(f)), _d(out))
        return out

    def dl_offsurf_direct(self, DEL, xq, nrm, area, g, xt, b, x0, n0, g0):
        nt = len(b)
        out = np.zeros(3 * nt)
        self.lib.or_dl_offsurf_direct(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                                      _d(_f64(area)), _d(_f64(g)), nt, _d(_f64(xt)), _d(_f64(b)),
                                      _d(_f64(x0)), _d(_f64(n0)), _d(_f64(g0)), _d(out))
        return out

    def dl_onsurf_direct(self, DEL, xq, nrm, area, g):
        out = np.zeros(3 * len(area))
        self.lib.or_dl_onsurf_direct(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                                     _d(_f64(area)), _d(_f64(g)), _d(out))
        return out

    def e2g_sl_away(self, xq, area, f, xt):
        nt = len(xt) // 3
        out = np.zeros(3 * nt)
        self.lib.or_e2g_sl_away(len(area), _d(_f64(xq)), _d(_f64(area)), _d(_f64(f)), nt,
                                _d(_f64(xt)), _d(out))
        return out

    def e2g_p_away(self, xq, area, f, xt):
        nt = len(xt) // 3
        out = np.zeros(nt)
        self.lib.or_e2g_p_away(len(area), _d(_f64(xq)), _d(_f64(area)), _d(_f64(f)), nt,
                               _d(_f64(xt)), _d(out))
        return out

    def e2g_sl_7ord(self, DEL, xq, nrm, area, f, xt, b, f0, n0):
        nt = len(b)
        out = np.zeros(3 * nt)
        self.lib.or_e2g_sl_7ord(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                                _d(_f64(area)), _d(_f64(f)), nt, _d(_f64(xt)), _d(_f64(b)),
                                _d(_f64(f0)), _d(_f64(n0)), _d(out))
        return out

    def e2g_p_7ord(self, DEL, xq, nrm, area, f, xt, b, f0, n0):
        nt = len(b)
        out = np.zeros(nt)
        self.lib.or_e2g_p_7ord(ctypes.c_double(DEL), len(area), _d(_f64(xq)), _d(_f64(nrm)),
                               _d(_f64(area)), _d(_f64(f)), nt, _d(_f64(xt)), _d(_f64(b)),
                               _d(_f64(f0)), _d(_f64(n0)), _d(out))
        return out

    # treecode -------------------------------------------------------------
    def kitc(self, kind, P, N0, theta, ctr, DEL, xq, nrm, area, dens, xt=None, b=None, x0=None,
             n0=None, dens0=None):
        """kind 0 SL on, 1 SL off, 2 DL on, 3 DL off. Returns (out, stats)."""
        if kind in (0, 2):
            xt = xq
        nt = len(xt) // 3
        out = np.zeros(3 * nt)
        stats = np.zeros(4, dtype=np.int64)
        self.lib.or_kitc_eval(kind, P, N0, ctypes.c_double(theta), _d(_f64(ctr)), ctypes.c_double(DEL),
                              len(area), _d(_f64(xq)), _d(_f64(nrm)), _d(_f64(area)), _d(_f64(dens)),
                              nt, _d(_f64(xt)), _d(None if b is None else _f64(b)),
                              _d(None if x0 is None else _f64(x0)), _d(None if n0 is None else _f64(n0)),
                              _d(None if dens0 is None else _f64(dens0)), _d(out),
                              stats.ctypes.data_as(_L))
        return out, stats

    def interp_dl_density(self, h, ctr, xq, g, nrst, x0, i123):
        nt = len(nrst)
        out = np.zeros(3 * nt)
        self.lib.or_interp_dl_density(ctypes.c_double(h), _d(_f64(ctr)), len(xq) // 3, _d(_f64(xq)),
                                      _d(_f64(g)), nt, _i(np.ascontiguousarray(nrst, np.int32)),
                                      _d(_f64(x0)), _i(np.ascontiguousarray(i123, np.int32)), _d(out))
        return out

    # two-surface scene ----------------------------------------------------
    class _Scene(ctypes.Structure):
        _fields_ = [("nq", ctypes.c_int * 2), ("xq", _D * 2), ("nrm", _D * 2), ("area", _D * 2),
                    ("ctr", (ctypes.c_double * 3) * 2), ("b", _D * 2), ("x0", _D * 2), ("n0", _D * 2),
                    ("nrst", _I * 2), ("i123", _I * 2), ("f0", _D * 2), ("h", ctypes.c_double),
                    ("DEL", ctypes.c_double), ("tree", ctypes.c_int), ("P", ctypes.c_int),
                    ("N0", ctypes.c_int), ("theta", ctypes.c_double)]

    def scene(self, geo: dict, tree=True, P=6, N0=1000, theta=0.6):
        """geo: dict with keys per surface s in (0,1): xq{s}, nrm{s}, area{s}, ctr{s},
        b{s}, x0{s}, n0{s}, nrst{s}, i123{s}, f0{s}; plus h, DEL."""
        keep = {}
        sc = Oracle._Scene()
        for s in (0, 1):
            for k in ("xq", "nrm", "area", "b", "x0", "n0", "f0"):
                keep[k + str(s)] = _f64(geo[k + str(s)])
            for k in ("nrst", "i123"):
                keep[k + str(s)] = np.ascontiguousarray(geo[k + str(s)], np.int32)
            sc.nq[s] = len(keep["area%d" % s])
            sc.xq[s] = _d(keep["xq%d" % s])
            sc.nrm[s] = _d(keep["nrm%d" % s])
            sc.area[s] = _d(keep["area%d" % s])
            for k in range(3):
                sc.ctr[s][k] = float(geo["ctr%d" % s][k])
            sc.b[s] = _d(keep["b%d" % s])
            sc.x0[s] = _d(keep["x0%d" % s])
            sc.n0[s] = _d(keep["n0%d" % s])
            sc.f0[s] = _d(keep["f0%d" % s])
            sc.nrst[s] = _i(keep["nrst%d" % s])
            sc.i123[s] = _i(keep["i123%d" % s])
        sc.h = geo["h"]
        sc.DEL = geo["DEL"]
        sc.tree = 1 if tree else 0
        sc.P = P
        sc.N0 = N0
        sc.theta = theta
        return sc, keep

    def matvec_2s(self, scene, u):
        sc, _keep = scene
        out = np.zeros_like(u)
        self.lib.or_matvec_2s(ctypes.byref(sc), _d(_f64(u)), _d(out))
        return out

    def rhs_2s(self, scene, f1, f2):
        sc, _keep = scene
        out = np.zeros(3 * (sc.nq[0] + sc.nq[1]))
        self.lib.or_rhs_2s(ctypes.byref(sc), _d(_f64(f1)), _d(_f64(f2)), _d(out))
        return out

    def gmres_2s(self, scene, b, x0=None, im=15, iter_max=100, tol=1e-10):
        sc, _keep = scene
        x = np.zeros(len(b)) if x0 is None else _f64(x0).copy()
        hist = np.zeros(iter_max + 1)
        it = self.lib.or_gmres_2s(ctypes.byref(sc), _d(_f64(b)), _d(x), im, iter_max,
                                  ctypes.c_double(tol), _d(hist))
        return x, hist[:it]

    # Poisson --------------------------------------------------------------
    def dst_poisson(self, n, f):
        a = _f64(f).copy()
        self.lib.or_dst_poisson(n, _d(a))
        return a

    def dst1_3d(self, n, f):
        a = _f64(f).copy()
        self.lib.or_dst1_3d(n, _d(a))
        return a

    def solve_poisson(self, N, L, h, band2_mask, out_mask, p, u, variable):
        uu = _f64(u).copy()
        self.lib.or_solve_poisson(N, ctypes.c_double(L), ctypes.c_double(h),
                                  _u8(np.ascontiguousarray(band2_mask, np.uint8)),
                                  _u8(np.ascontiguousarray(out_mask, np.uint8)), _d(_f64(p)), _d(uu),
                                  variable)
        return uu


def ref_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "librefe2g.so"))


class Ref2S:
    """The unmodified reference two-surface program (oracle/_ref)."""

    def __init__(self, P=6, N0=1000):
        path = os.path.join(REF_DIR, "libref2s_P%d_N%d.so" % (P, N0))
        self.lib = ctypes.CDLL(path)
        self.lib.ref2s_solve.restype = ctypes.c_int
        self.lib.ref2s_log.restype = ctypes.c_char_p
        self.P, self.N0 = P, N0

    def setup(self, N):
        self.lib.ref2s_setup(N)
        a, b = ctypes.c_int(), ctypes.c_int()
        h, d = ctypes.c_double(), ctypes.c_double()
        self.lib.ref2s_counts(ctypes.byref(a), ctypes.byref(b), ctypes.byref(h), ctypes.byref(d))
        self.nq = (a.value, b.value)
        self.h, self.DEL = h.value, d.value
        return self

    def surface(self, s):
        n = self.nq[s]
        xyz, nrm, f, g = (np.zeros(3 * n) for _ in range(4))
        area = np.zeros(n)
        plane = np.zeros(n, np.int32)
        self.lib.ref2s_get_surface(s, _d(xyz), _d(nrm), _d(area), _i(plane), _d(f), _d(g))
        return dict(xq=xyz, nrm=nrm, area=area, plane=plane, f=f, g=g)

    def targets(self, t):
        n = self.nq[t]
        b = np.zeros(n)
        x0, n0, f0, g0 = (np.zeros(3 * n) for _ in range(4))
        nrst = np.zeros(n, np.int32)
        i123 = np.zeros(3 * n, np.int32)
        self.lib.ref2s_get_targets(t, _d(b), _d(x0), _d(n0), _d(f0), _d(g0), _i(nrst), _i(i123))
        return dict(b=b, x0=x0, n0=n0, f0=f0, g0=g0, nrst=nrst, i123=i123)

    def set_f(self, s, f):
        self.lib.ref2s_set_f(s, _d(_f64(f)))

    def set_g(self, s, g):
        self.lib.ref2s_set_g(s, _d(_f64(g)))

    def set_nrst_g(self, t, g0):
        self.lib.ref2s_set_nrst_g(t, _d(_f64(g0)))

    def interpolate(self, s):
        self.lib.ref2s_interpolate(s)

    def eval(self, kind, tree, s, t):
        out = np.zeros(3 * self.nq[t])
        self.lib.ref2s_eval(kind, 1 if tree else 0, s, t, _d(out))
        return out

    def rhs(self):
        out = np.zeros(3 * sum(self.nq))
        self.lib.ref2s_rhs(_d(out))
        return out

    def matvec(self, u):
        out = np.zeros(3 * sum(self.nq))
        self.lib.ref2s_matvec(_d(_f64(u)), _d(out))
        return out

    def solve(self):
        x = np.zeros(3 * sum(self.nq))
        r = np.zeros(400)
        k = self.lib.ref2s_solve(_d(x), _d(r), 400)
        return x, r[:k]

    def load(self, geo: dict, g=None):
        """Loads a scene in the oracle's dict layout (see Oracle.scene) into
        the reference program instead of its own set-up; g (optional, per
        surface) is the stresslet density."""
        for s in (0, 1):
            n = len(geo["area%d" % s])
            gs = np.zeros(3 * n) if g is None else _f64(g[s])
            self.lib.ref2s_load(s, n, _d(_f64(geo["xq%d" % s])), _d(_f64(geo["nrm%d" % s])),
                                _d(_f64(geo["area%d" % s])), _d(_f64(geo["f%d" % s])), _d(gs),
                                _d(_f64(geo["b%d" % s])), _d(_f64(geo["x0%d" % s])), _d(_f64(geo["n0%d" % s])),
                                _d(_f64(geo["f0%d" % s])), _i(np.ascontiguousarray(geo["nrst%d" % s], np.int32)),
                                _i(np.ascontiguousarray(geo["i123%d" % s], np.int32)), ctypes.c_double(geo["h"]),
                                ctypes.c_double(geo["DEL"]))
        self.nq = tuple(len(geo["area%d" % s]) for s in (0, 1))
        self.h, self.DEL = float(geo["h"]), float(geo["DEL"])
        return self

    def sample_eval(self, kind, s, t, idx):
        """Direct sums (kind 0 Stokeslet of f, 1 stresslet of g) of surface s
        at the sampled targets idx of set t, by the reference's own functions;
        returns (out (3 per target), g0 at the targets' nearest points (the
        stresslet off the surface only, else None))."""
        idx = np.ascontiguousarray(idx, np.int32)
        out = np.zeros(3 * len(idx))
        g0 = np.zeros(3 * len(idx)) if (kind == 1 and s != t) else None
        self.lib.ref2s_sample_eval(kind, s, t, len(idx), _i(idx), _d(out), _d(g0))
        return out, g0

    def geometry(self):
        """Scene geometry in the oracle's dict layout (see Oracle.scene)."""
        ctrs = [(0.0, 0.0, -0.5 - 1.0 / 4096.0), (0.0, 0.0, 0.5)]
        geo = dict(h=self.h, DEL=self.DEL)
        for s in (0, 1):
            S = self.surface(s)
            T = self.targets(s)
            geo.update({"xq%d" % s: S["xq"], "nrm%d" % s: S["nrm"], "area%d" % s: S["area"],
                        "plane%d" % s: S["plane"], "f%d" % s: S["f"], "ctr%d" % s: np.array(ctrs[s]),
                        "b%d" % s: T["b"], "x0%d" % s: T["x0"], "n0%d" % s: T["n0"],
                        "f0%d" % s: T["f0"], "nrst%d" % s: T["nrst"], "i123%d" % s: T["i123"]})
        return geo


class RefE2G:
    """The unmodified reference extend-to-grid program (oracle/_ref)."""

    def __init__(self):
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, "librefe2g.so"))
        self.lib.refe2g_log.restype = ctypes.c_char_p
        self.lib.refe2g_p_exact.restype = ctypes.c_double

    def setup(self, N):
        self.N = N
        self.lib.refe2g_setup(N)
        a, b = ctypes.c_int(), ctypes.c_int()
        h, d = ctypes.c_double(), ctypes.c_double()
        self.lib.refe2g_counts(ctypes.byref(a), ctypes.byref(b), ctypes.byref(h), ctypes.byref(d))
        self.nq, self.nt, self.h, self.DEL = a.value, b.value, h.value, d.value
        return self

    def log(self):
        return self.lib.refe2g_log().decode()

    def surface(self):
        n = self.nq
        xyz, nrm, f = (np.zeros(3 * n) for _ in range(3))
        area = np.zeros(n)
        self.lib.refe2g_get_surface(_d(xyz), _d(nrm), _d(area), _d(f))
        return dict(xq=xyz, nrm=nrm, area=area, f=f)

    def targets(self):
        n = self.nt
        b = np.zeros(n)
        x0, n0 = np.zeros(3 * n), np.zeros(3 * n)
        band2 = np.zeros(n, np.int32)
        self.lib.refe2g_get_targets(_d(b), _d(x0), _d(n0), _i(band2))
        return dict(b=b, x0=x0, n0=n0, band2=band2)

    def nrst(self):
        m = (self.N + 1) ** 3
        a = np.zeros(m, np.int32)
        self.lib.refe2g_get_nrst(_i(a))
        return a

    def grid_zeros(self):
        return np.zeros((self.N + 1) ** 3)

    def eval_p_faces(self):
        p = self.grid_zeros()
        self.lib.refe2g_eval_p_faces(_d(p))
        return p

    def eval_p_band(self, p):
        p = _f64(p).copy()
        self.lib.refe2g_eval_p_band(_d(p))
        return p

    def eval_u_faces(self):
        u = [self.grid_zeros() for _ in range(3)]
        self.lib.refe2g_eval_u_faces(*[_d(a) for a in u])
        return u

    def eval_u_band(self, u):
        u = [_f64(a).copy() for a in u]
        self.lib.refe2g_eval_u_band(*[_d(a) for a in u])
        return u

    def solve_poisson(self, variable, p, u):
        u = _f64(u).copy()
        self.lib.refe2g_solve_poisson(variable, _d(_f64(p)), _d(u))
        return u

    def dst_poisson(self, n, f):
        a = _f64(f).copy()
        self.lib.refe2g_dst_poisson(n, _d(a))
        return a

    def run(self):
        """The whole reference driver at the set-up grid; returns its printed
        output (this run's only)."""
        self.lib.refe2g_clear_log()
        self.lib.refe2g_run()
        return self.log()

    def load(self, N, scene):
        """Loads an extend-to-grid scene (the dict of the product's
        E2G.scene(): quadrature, density, tagged targets, index grid)
        instead of the reference's own set-up."""
        self.N = N
        nq, nt = len(scene["area"]), len(scene["b"])
        self.lib.refe2g_load(N, nq, _d(_f64(scene["xq"])), _d(_f64(scene["nrm"])), _d(_f64(scene["area"])),
                             _d(_f64(scene["f"])), nt, _d(_f64(scene["b"])), _d(_f64(scene["x0"])),
                             _d(_f64(scene["n0"])), _i(np.ascontiguousarray(scene["band2"], np.int32)),
                             _i(np.ascontiguousarray(scene["nrst"], np.int32)))
        self.nq, self.nt = nq, nt
        h = 3.0 / N
        self.h = h
        return self

    def set_nrst(self, nrst_grid):
        self.lib.refe2g_set_nrst(_i(np.ascontiguousarray(nrst_grid, np.int32)))

    def away_points(self, xyz):
        """The reference's plain Stokeslet and pressure sums at points xyz
        (3 per point): returns (u (3 per point), p)."""
        xyz = _f64(xyz)
        n = len(xyz) // 3
        u, p = np.zeros(3 * n), np.zeros(n)
        self.lib.refe2g_away_points(n, _d(xyz), _d(u), _d(p))
        return u, p

    def p_exact(self, x, y, z):
        return self.lib.refe2g_p_exact(ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z))

    def u_exact(self, x, y, z):
        u = np.zeros(3)
        self.lib.refe2g_u_exact(ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z), _d(u))
        return u
