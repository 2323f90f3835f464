"""Python front end of libhighreg_b200.so (ctypes over include/highreg_b200.h).

The CUDA library is the only compute path: if it cannot be loaded, or no
sm_100 GPU is present, the calls raise instead of falling back to anything.

Array conventions follow the reference: points and vector fields are
interleaved xyz float64 arrays (v[3*j+k]); scene dictionaries use the keys
``xq{s} nrm{s} area{s} plane{s} ctr{s} f{s} b{s} x0{s} n0{s} f0{s} nrst{s}
i123{s}`` for surface s in (0, 1) plus ``h`` and ``DEL``.
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhighreg_b200.so")

HR_OK, HR_ERR_ARG, HR_ERR_CUDA, HR_ERR_NAN, HR_ERR_NOT_CONVERGED, HR_ERR_NO_DEVICE, HR_ERR_STATE = range(7)
HR_DIRECT, HR_TREE = 0, 1
HR_FP64, HR_MIXED, HR_FP32 = 0, 1, 2

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_U8 = ctypes.POINTER(ctypes.c_uint8)


class HrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("highreg error %d: %s" % (code, msg))
        self.code = code


class Surface(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("xyz", _D), ("nrml", _D), ("area", _D), ("plane", _I),
                ("center", ctypes.c_double * 3)]


class Targets(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("xyz", _D), ("b", _D), ("x0", _D), ("n0", _D), ("nrst", _I),
                ("i123", _I)]


class EvalOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("P", ctypes.c_int), ("N0", ctypes.c_int),
                ("theta", ctypes.c_double), ("precision", ctypes.c_int)]


class Scene2S(ctypes.Structure):
    _fields_ = [("surf", Surface * 2), ("tgt", Targets * 2), ("f0", _D * 2), ("h", ctypes.c_double),
                ("delta", ctypes.c_double)]


class GmresOpts(ctypes.Structure):
    _fields_ = [("restart", ctypes.c_int), ("max_iter", ctypes.c_int), ("tol", ctypes.c_double),
                ("precision", ctypes.c_int), ("use_guess", ctypes.c_int), ("true_residual", ctypes.c_int),
                ("mixed_accuracy", ctypes.c_double)]


class GmresReport(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("restarts", ctypes.c_int), ("matvecs_fp64", ctypes.c_int),
                ("matvecs_mixed", ctypes.c_int), ("residual", ctypes.c_double),
                ("true_residual", ctypes.c_double), ("seconds", ctypes.c_double),
                ("guess_rejected", ctypes.c_int), ("resid_hist", ctypes.c_double * 512)]

    def as_dict(self):
        return dict(iterations=self.iterations, restarts=self.restarts, matvecs_fp64=self.matvecs_fp64,
                    matvecs_mixed=self.matvecs_mixed, residual=self.residual,
                    true_residual=self.true_residual, seconds=self.seconds,
                    guess_rejected=self.guess_rejected,
                    resid_hist=[self.resid_hist[i] for i in range(min(self.iterations, 512))])


class Work(ctypes.Structure):
    _fields_ = [("direct_pairs_near", ctypes.c_longlong), ("direct_pairs_far", ctypes.c_longlong),
                ("proxy_pairs", ctypes.c_longlong), ("moment_terms", ctypes.c_longlong),
                ("flops", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Geom2SParams(ctypes.Structure):
    _fields_ = [("axes", ctypes.c_double * 3), ("center", (ctypes.c_double * 3) * 2),
                ("unrot", (ctypes.c_double * 9) * 2), ("rotated", ctypes.c_int * 2),
                ("kappa0", ctypes.c_double), ("q", ctypes.c_double), ("tension_body", ctypes.c_int)]


_lib = None


def lib():
    """Loads the in-tree CUDA library (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HrError(HR_ERR_STATE, "libhighreg_b200.so not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        L.hr_last_error.restype = ctypes.c_char_p
        L.hr_ctx_launch_count.restype = ctypes.c_longlong
        L.hr_plan2s_stream.restype = ctypes.c_void_p
        L.hr_geom2s_destroy.restype = None
        L.hr_plan2s_destroy.restype = None
        L.hr_ctx_destroy.restype = None
        L.hr_dst1_plan_destroy.restype = None
        L.hr_host_free.restype = None
        L.hr_host_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def pinned_empty(n, dtype=np.float64):
    """An uninitialised 1-D numpy array of n elements in page-locked host memory
    (hr_host_alloc), freed with the array. Copies between it and the device run
    at DMA speed, without the staging that pageable memory needs."""
    dtype = np.dtype(dtype)
    nbytes = max(1, int(n) * dtype.itemsize)
    ptr = ctypes.c_void_p()
    rc = lib().hr_host_alloc(ctypes.c_size_t(nbytes), ctypes.byref(ptr))
    if rc != HR_OK:
        raise HrError(rc, "hr_host_alloc of %d bytes failed" % nbytes)
    buf = (ctypes.c_char * nbytes).from_address(ptr.value)
    arr = np.frombuffer(buf, dtype=dtype, count=int(n))
    weakref.finalize(buf, lib().hr_host_free, ptr.value)
    return arr


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


def _devp(t):
    """Device pointer of a torch CUDA tensor as a double*."""
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), _D)


class _Keep:
    """Keeps numpy arrays alive while a ctypes struct points at them."""

    def __init__(self):
        self.arrs = []

    def f(self, a):
        if a is None:
            return None
        a = _f64(a)
        self.arrs.append(a)
        return a

    def i(self, a):
        if a is None:
            return None
        a = _i32(a)
        self.arrs.append(a)
        return a


def make_surface(keep, xq, nrm, area, plane=None, ctr=(0.0, 0.0, 0.0)):
    s = Surface()
    xq, nrm, area = keep.f(xq), keep.f(nrm), keep.f(area)
    plane = keep.i(plane)
    s.n = len(area)
    s.xyz, s.nrml, s.area, s.plane = _dp(xq), _dp(nrm), _dp(area), _ip(plane)
    for k in range(3):
        s.center[k] = float(ctr[k])
    return s


def make_targets(keep, xyz, b=None, x0=None, n0=None, nrst=None, i123=None):
    t = Targets()
    xyz = keep.f(xyz)
    t.n = len(xyz) // 3
    t.xyz = _dp(xyz)
    t.b = _dp(keep.f(b))
    t.x0 = _dp(keep.f(x0))
    t.n0 = _dp(keep.f(n0))
    t.nrst = _ip(keep.i(nrst))
    t.i123 = _ip(keep.i(i123))
    return t


def eval_opts(mode=HR_TREE, P=6, N0=1000, theta=0.6, precision=HR_FP64):
    o = EvalOpts()
    o.mode, o.P, o.N0, o.theta, o.precision = mode, P, N0, theta, precision
    return o


class Context:
    """A CUDA context of the library (one stream)."""

    def __init__(self, device: int = 0):
        L = lib()
        p = ctypes.c_void_p()
        rc = L.hr_ctx_create(device, ctypes.byref(p))
        if rc != HR_OK:
            raise HrError(rc, "hr_ctx_create failed (no sm_100 device?)")
        self.p = p
        self._children = weakref.WeakSet()

    def adopt(self, obj):
        """Registers an object (plan, pipeline, network) that closes with the context."""
        self._children.add(obj)

    def close(self):
        """Closes the objects made on this context, then the context itself."""
        if self.p:
            for obj in list(getattr(self, "_children", ())):
                obj.close()
            lib().hr_ctx_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != HR_OK:
            raise HrError(rc, lib().hr_last_error(self.p).decode())

    @property
    def launches(self):
        return lib().hr_ctx_launch_count(self.p)

    # ---- drop-in boundary sums
    def sl_onsurf(self, DEL, xq, nrm, area, f, ctr=(0, 0, 0), **opt):
        k = _Keep()
        S = make_surface(k, xq, nrm, area, ctr=ctr)
        o = eval_opts(**opt)
        out = np.zeros(3 * S.n)
        self._check(lib().hr_stokes_sl_onsurf(self.p, ctypes.byref(o), ctypes.c_double(DEL), ctypes.byref(S),
                                              _dp(k.f(f)), _dp(out)))
        return out

    def sl_offsurf(self, DEL, xq, nrm, area, f, xt, b, n0, f0, ctr=(0, 0, 0), **opt):
        k = _Keep()
        S = make_surface(k, xq, nrm, area, ctr=ctr)
        T = make_targets(k, xt, b=b, n0=n0)
        o = eval_opts(**opt)
        out = np.zeros(3 * T.n)
        self._check(lib().hr_stokes_sl_offsurf(self.p, ctypes.byref(o), ctypes.c_double(DEL), ctypes.byref(S),
                                               _dp(k.f(f)), ctypes.byref(T), _dp(k.f(f0)), _dp(out)))
        return out

    def dl_onsurf(self, DEL, xq, nrm, area, g, ctr=(0, 0, 0), **opt):
        k = _Keep()
        S = make_surface(k, xq, nrm, area, ctr=ctr)
        o = eval_opts(**opt)
        out = np.zeros(3 * S.n)
        self._check(lib().hr_stokes_dl_onsurf(self.p, ctypes.byref(o), ctypes.c_double(DEL), ctypes.byref(S),
                                              _dp(k.f(g)), _dp(out)))
        return out

    def dl_offsurf(self, DEL, xq, nrm, area, g, xt, b, x0, n0, g0, ctr=(0, 0, 0), **opt):
        k = _Keep()
        S = make_surface(k, xq, nrm, area, ctr=ctr)
        T = make_targets(k, xt, b=b, x0=x0, n0=n0)
        o = eval_opts(**opt)
        out = np.zeros(3 * T.n)
        self._check(lib().hr_stokes_dl_offsurf(self.p, ctypes.byref(o), ctypes.c_double(DEL), ctypes.byref(S),
                                               _dp(k.f(g)), ctypes.byref(T), _dp(k.f(g0)), _dp(out)))
        return out

    def interpolate_dl_density(self, h, xq, g, ctr, plane, x0, nrst, i123):
        k = _Keep()
        nq = len(xq) // 3
        S = make_surface(k, xq, np.zeros(3 * nq), np.zeros(nq), plane=plane, ctr=ctr)
        T = make_targets(k, x0, x0=x0, nrst=nrst, i123=i123)
        out = np.zeros(3 * T.n)
        self._check(lib().hr_interpolate_dl_density(self.p, ctypes.c_double(h), ctypes.byref(S), _dp(k.f(g)),
                                                    ctypes.byref(T), _dp(out)))
        return out

    # ---- extend-to-grid
    def e2g_sl_away(self, xq, area, f, xt):
        k = _Keep()
        nq = len(area)
        S = make_surface(k, xq, np.zeros(3 * nq), area)
        xt = k.f(xt)
        out = np.zeros(len(xt))
        self._check(lib().hr_e2g_stokeslet_away(self.p, ctypes.byref(S), _dp(k.f(f)), len(xt) // 3, _dp(xt),
                                                _dp(out)))
        return out

    def e2g_p_away(self, xq, area, f, xt):
        k = _Keep()
        nq = len(area)
        S = make_surface(k, xq, np.zeros(3 * nq), area)
        xt = k.f(xt)
        out = np.zeros(len(xt) // 3)
        self._check(lib().hr_e2g_pressure_away(self.p, ctypes.byref(S), _dp(k.f(f)), len(xt) // 3, _dp(xt),
                                               _dp(out)))
        return out

    def e2g_sl_7ord(self, DEL, xq, nrm, area, f, xt, b, f0, n0):
        k = _Keep()
        S = make_surface(k, xq, nrm, area)
        T = make_targets(k, xt, b=b, n0=n0)
        out = np.zeros(3 * T.n)
        self._check(lib().hr_e2g_stokeslet_7ord(self.p, ctypes.c_double(DEL), ctypes.byref(S), _dp(k.f(f)),
                                                ctypes.byref(T), _dp(k.f(f0)), _dp(out)))
        return out

    def e2g_p_7ord(self, DEL, xq, nrm, area, f, xt, b, f0, n0):
        k = _Keep()
        S = make_surface(k, xq, nrm, area)
        T = make_targets(k, xt, b=b, n0=n0)
        out = np.zeros(T.n)
        self._check(lib().hr_e2g_pressure_7ord(self.p, ctypes.c_double(DEL), ctypes.byref(S), _dp(k.f(f)),
                                               ctypes.byref(T), _dp(k.f(f0)), _dp(out)))
        return out

    def dst_poisson3d(self, n, f):
        a = _f64(f).copy()
        self._check(lib().hr_dst_poisson3d(self.p, n, _dp(a)))
        return a

    def dst1_3d(self, n, f):
        """The plain 3D DST-I (FFTW's RODFT00 on all three axes, unnormalised) of
        a row-major n^3 array, through a reusable plan (hr_dst1_*)."""
        L = lib()
        plan = ctypes.c_void_p()
        self._check(L.hr_dst1_plan_create(self.p, n, ctypes.byref(plan)))
        a = _f64(f)
        out = np.empty_like(a)
        try:
            self._check(L.hr_dst1_execute(plan, _dp(a), _dp(out)))
        finally:
            L.hr_dst1_plan_destroy(plan)
        return out

    def solve_poisson(self, N, L, band2, outside, p, u, variable):
        band2 = np.ascontiguousarray(band2, np.uint8)
        outside = np.ascontiguousarray(outside, np.uint8)
        p = None if p is None else _f64(p)
        uu = _f64(u).copy()
        self._check(lib().hr_e2g_solve_poisson(self.p, N, ctypes.c_double(L), band2.ctypes.data_as(_U8),
                                               outside.ctypes.data_as(_U8), _dp(p), _dp(uu), variable))
        return uu

    def fp64_peak(self):
        v = ctypes.c_double()
        self._check(lib().hr_measure_fp64_peak(self.p, ctypes.byref(v)))
        return v.value

    def fp32_peak(self):
        v = ctypes.c_double()
        self._check(lib().hr_measure_fp32_peak(self.p, ctypes.byref(v)))
        return v.value


class Geometry2S:
    """The product's two-surface scene generator (host C++)."""

    def __init__(self, N: int, params: Geom2SParams | None = None):
        L = lib()
        if params is None:
            params = Geom2SParams()
            L.hr_geom2s_default_params(ctypes.byref(params))
        self.params = params
        p = ctypes.c_void_p()
        rc = L.hr_geom2s_generate(ctypes.byref(params), N, ctypes.byref(p))
        if rc != HR_OK:
            raise HrError(rc, "hr_geom2s_generate failed")
        self.p = p
        sc = Scene2S()
        force = (_D * 2)()
        L.hr_geom2s_view(p, ctypes.byref(sc), force)
        d = dict(h=sc.h, DEL=sc.delta)
        for s in (0, 1):
            S, T = sc.surf[s], sc.tgt[s]
            n = S.n
            d["xq%d" % s] = np.ctypeslib.as_array(S.xyz, (3 * n,)).copy()
            d["nrm%d" % s] = np.ctypeslib.as_array(S.nrml, (3 * n,)).copy()
            d["area%d" % s] = np.ctypeslib.as_array(S.area, (n,)).copy()
            d["plane%d" % s] = np.ctypeslib.as_array(S.plane, (n,)).copy()
            d["ctr%d" % s] = np.array([S.center[k] for k in range(3)])
            d["f%d" % s] = np.ctypeslib.as_array(force[s], (3 * n,)).copy()
            d["b%d" % s] = np.ctypeslib.as_array(T.b, (n,)).copy()
            d["x0%d" % s] = np.ctypeslib.as_array(T.x0, (3 * n,)).copy()
            d["n0%d" % s] = np.ctypeslib.as_array(T.n0, (3 * n,)).copy()
            d["f0%d" % s] = np.ctypeslib.as_array(sc.f0[s], (3 * n,)).copy()
            d["nrst%d" % s] = np.ctypeslib.as_array(T.nrst, (n,)).copy()
            d["i123%d" % s] = np.ctypeslib.as_array(T.i123, (3 * n,)).copy()
        self.scene = d
        ph = (ctypes.c_double * 4)()
        L.hr_geom2s_phase_seconds(p, ph)
        # wall seconds of the set-up phases: quadrature, forces, nearest data of sets 0 and 1
        self.phase_seconds = {"quadrature": ph[0], "forces": ph[1], "nearest0": ph[2], "nearest1": ph[3]}
        L.hr_geom2s_destroy(p)
        self.p = None

    @staticmethod
    def default_params():
        p = Geom2SParams()
        lib().hr_geom2s_default_params(ctypes.byref(p))
        return p


def scene_struct(keep, geo):
    sc = Scene2S()
    for s in (0, 1):
        sc.surf[s] = make_surface(keep, geo["xq%d" % s], geo["nrm%d" % s], geo["area%d" % s],
                                  plane=geo["plane%d" % s], ctr=geo["ctr%d" % s])
        sc.tgt[s] = make_targets(keep, geo["xq%d" % s], b=geo["b%d" % s], x0=geo["x0%d" % s],
                                 n0=geo["n0%d" % s], nrst=geo["nrst%d" % s], i123=geo["i123%d" % s])
        sc.f0[s] = _dp(keep.f(geo["f0%d" % s]))
    sc.h = geo["h"]
    sc.delta = geo["DEL"]
    return sc


def gmres_opts(restart=15, max_iter=100, tol=1e-10, precision=HR_FP64, use_guess=False, true_residual=False,
               mixed_accuracy=0.0):
    o = GmresOpts()
    o.restart, o.max_iter, o.tol, o.precision = restart, max_iter, tol, precision
    o.use_guess, o.true_residual = int(bool(use_guess)), int(bool(true_residual))
    o.mixed_accuracy = mixed_accuracy
    return o


def write_npy(path, a):
    """Writes a float64 array as a .npy file through the library's writer (hr_write_npy)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    shape = (ctypes.c_longlong * max(1, a.ndim))(*(a.shape or (1,)))
    rc = lib().hr_write_npy(str(path).encode(), _dp(a), max(1, a.ndim), shape)
    if rc != HR_OK:
        raise HrError(rc, "hr_write_npy failed for %s" % path)


class Plan2S:
    """Device-resident two-surface problem (trees, lists, stencils uploaded once)."""

    def __init__(self, ctx: Context, geo: dict, **opt):
        self.ctx = ctx
        ctx.adopt(self)
        self.keep = _Keep()
        sc = scene_struct(self.keep, geo)
        self.opts = eval_opts(**opt)
        p = ctypes.c_void_p()
        ctx._check(lib().hr_plan2s_create(ctx.p, ctypes.byref(sc), ctypes.byref(self.opts), ctypes.byref(p)))
        self.p = p
        self.n = 3 * (len(geo["area0"]) + len(geo["area1"]))
        self.n1 = len(geo["area0"])

    def close(self):
        if getattr(self, "p", None):
            lib().hr_plan2s_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def matvec(self, x):
        x = _f64(x)
        y = np.zeros(self.n)
        self.ctx._check(lib().hr_plan2s_matvec(self.p, _dp(x), _dp(y)))
        return y

    def rhs(self, f1, f2):
        b = np.zeros(self.n)
        self.ctx._check(lib().hr_plan2s_rhs(self.p, _dp(_f64(f1)), _dp(_f64(f2)), _dp(b)))
        return b

    def solve(self, b, x0=None, check=True, **gopt):
        x = np.zeros(self.n) if x0 is None else _f64(x0).copy()
        o = gmres_opts(use_guess=x0 is not None, **gopt)
        rep = GmresReport()
        rc = lib().hr_plan2s_solve(self.p, ctypes.byref(o), _dp(_f64(b)), _dp(x), ctypes.byref(rep))
        if check:
            self.ctx._check(rc)
        return x, rep.as_dict()

    def work(self, which=0):
        """Work counts: 0 one matvec (counted by a launch), 1 the RHS, 2 the inner
        treecode's stresslet batch (from its lists; flops 0)."""
        w = Work()
        self.ctx._check(lib().hr_plan2s_work(self.p, which, ctypes.byref(w)))
        return w.as_dict()

    # device-resident variants (torch CUDA float64 tensors)
    def matvec_dev(self, x, y, precision=HR_FP64):
        self.ctx._check(lib().hr_plan2s_matvec_dev(self.p, _devp(x), _devp(y), precision))

    def rhs_dev(self, f1, f2, b):
        self.ctx._check(lib().hr_plan2s_rhs_dev(self.p, _devp(f1), _devp(f2), _devp(b)))

    def solve_dev(self, b, x, use_guess=False, check=True, **gopt):
        o = gmres_opts(use_guess=use_guess, **gopt)
        rep = GmresReport()
        rc = lib().hr_plan2s_solve_dev(self.p, ctypes.byref(o), _devp(b), _devp(x), ctypes.byref(rep))
        if check:
            self.ctx._check(rc)
        return rep.as_dict()

    def stream(self):
        return lib().hr_plan2s_stream(self.p)

    def check_upward_pass(self, x):
        """Max relative difference of the tensor-core (3xTF32) moments from the FP64 ones."""
        v = ctypes.c_double()
        self.ctx._check(lib().hr_plan2s_check_upward_pass(self.p, _dp(_f64(x)), ctypes.byref(v)))
        return v.value

    def set_inner_tree(self, P, N0, theta=0.6):
        """Own treecode (degree P, leaf size N0, MAC theta) for the reduced-precision
        inner operator of GMRES-IR; P = 0 removes it. FP64 true residuals keep the
        plan's treecode. Returns the inner operator's measured relative L2 error
        (0 when removed), the default mixed_accuracy of later solves."""
        e = ctypes.c_double(0.0)
        self.ctx._check(lib().hr_plan2s_set_inner_tree(self.p, int(P), int(N0), ctypes.c_double(theta),
                                                       ctypes.byref(e)))
        return e.value

    def time_batch(self, which=0, iters=10):
        """Milliseconds per launch of one boundary-sum batch (0 DL fp64, 1 SL, 2 DL mixed,
        3 DL mixed on the inner treecode)."""
        v = ctypes.c_double()
        self.ctx._check(lib().hr_plan2s_time_batch(self.p, which, iters, ctypes.byref(v)))
        return v.value


class E2GErrors(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("p_max", "p_rms", "u_max", "u_rms", "band_u_max", "band_u_rms",
                                                "ref_p_max_rel", "ref_p_rel_l2", "ref_u_max_rel", "ref_u_rel_l2")]


class E2GInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("L", ctypes.c_double), ("h", ctypes.c_double), ("delta", ctypes.c_double),
                ("nq", ctypes.c_int), ("n_tagged", ctypes.c_int), ("n_band", ctypes.c_int), ("n_face", ctypes.c_int),
                ("pairs", ctypes.c_longlong)]


class E2GReport(ctypes.Structure):
    _fields_ = [("seconds_sums", ctypes.c_double), ("seconds_poisson", ctypes.c_double),
                ("seconds_total", ctypes.c_double), ("pairs", ctypes.c_longlong)]


class E2G:
    """The extend-to-grid pipeline (translating spheroid, h = 3/N) on the device."""

    def __init__(self, ctx: Context, N: int):
        self.ctx = ctx
        ctx.adopt(self)
        p = ctypes.c_void_p()
        ctx._check(lib().hr_e2g_create(ctx.p, N, ctypes.byref(p)))
        self.p = p
        info = E2GInfo()
        lib().hr_e2g_get_info(p, ctypes.byref(info))
        self.info = {k: getattr(info, k) for k, _ in E2GInfo._fields_}
        self.N = N

    def close(self):
        if getattr(self, "p", None):
            lib().hr_e2g_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def snapshot(self):
        """Keeps the current extended grids as the reference of error_norms."""
        self.ctx._check(lib().hr_e2g_snapshot(self.p))

    def error_norms(self):
        e = E2GErrors()
        self.ctx._check(lib().hr_e2g_error_norms(self.p, ctypes.byref(e)))
        return {k: getattr(e, k) for k, _ in E2GErrors._fields_}

    def run(self, precision=HR_FP64):
        rep = E2GReport()
        self.ctx._check(lib().hr_e2g_run(self.p, precision, ctypes.byref(rep)))
        return {k: getattr(rep, k) for k, _ in E2GReport._fields_}

    def get(self, which, out=None):
        """Grid `which` of the last run (hr_e2g_get) as float64. `out`, if
        given (e.g. from pinned_empty), is filled in place and returned."""
        m = (self.N + 1) ** 3
        n = 3 * m if which in (1, 3) else m
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise HrError(HR_ERR_ARG, "E2G.get: out must be a contiguous float64 array of %d elements" % n)
        self.ctx._check(lib().hr_e2g_get(self.p, which, _dp(out)))
        return out

    def midplane(self):
        """Mid-plane y = 1.5 slices of the last run, shape (4, N+1, N+1) in (i, k) order:
        extended p, |p - p_exact|, |u - u_exact| (0 inside the body) and p_exact (0 inside)."""
        M = self.N + 1
        out = np.zeros(4 * M * M)
        self.ctx._check(lib().hr_e2g_midplane(self.p, _dp(out)))
        return out.reshape(4, M, M)

    def scene(self):
        nq, nt = self.info["nq"], self.info["n_tagged"]
        q = np.zeros(10 * nq)
        lib().hr_e2g_scene(self.p, 0, q.ctypes.data_as(ctypes.c_void_p))
        nrst = np.zeros((self.N + 1) ** 3, np.int32)
        lib().hr_e2g_scene(self.p, 1, nrst.ctypes.data_as(ctypes.c_void_p))
        t = np.zeros(8 * nt)
        lib().hr_e2g_scene(self.p, 2, t.ctypes.data_as(ctypes.c_void_p))
        return dict(xq=q[:3 * nq], nrm=q[3 * nq:6 * nq], area=q[6 * nq:7 * nq], f=q[7 * nq:10 * nq], nrst=nrst,
                    b=t[:nt], x0=t[nt:4 * nt], n0=t[4 * nt:7 * nt], band2=t[7 * nt:].astype(np.int32))


def e2g_exact(x, y, z):
    """Exact pressure and velocity of the translating spheroid at one point."""
    L = lib()
    L.hr_e2g_p_exact.restype = ctypes.c_double
    u = np.zeros(3)
    L.hr_e2g_u_exact(ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z), _dp(u))
    return L.hr_e2g_p_exact(ctypes.c_double(x), ctypes.c_double(y), ctypes.c_double(z)), u


# ---------------------------------------------------------------- warm start
NFEAT = 12


class WarmInstance(ctypes.Structure):
    _fields_ = [("geom", Geom2SParams), ("U", ctypes.c_double * 3), ("Omega", ctypes.c_double * 3),
                ("xmid", ctypes.c_double * 3), ("gap", ctypes.c_double)]

    def as_dict(self):
        return dict(U=list(self.U), Omega=list(self.Omega), xmid=list(self.xmid), gap=self.gap,
                    center2=list(self.geom.center[1]), unrot2=list(self.geom.unrot[1]))


def warm_instance(seed: int, index: int) -> WarmInstance:
    """Seeded two-surface instance (random gap, orientation, rigid motion)."""
    w = WarmInstance()
    rc = lib().hr_warm_instance_make(ctypes.c_ulonglong(seed), index, ctypes.byref(w))
    if rc != HR_OK:
        raise HrError(rc, "hr_warm_instance_make failed")
    return w


def warm_features(geo: dict, inst: WarmInstance):
    """(features float32 [n, 12], imposed velocity float64 [3n]) of a scene."""
    keep = _Keep()
    sc = scene_struct(keep, geo)
    n = len(geo["area0"]) + len(geo["area1"])
    feat = np.zeros((n, NFEAT), np.float32)
    u = np.zeros(3 * n)
    rc = lib().hr_warm_features(ctypes.byref(sc), ctypes.byref(inst),
                                feat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _dp(u))
    if rc != HR_OK:
        raise HrError(rc, "hr_warm_features failed")
    return feat, u


def warm_frames(inst: WarmInstance):
    """Body frames of the two surfaces: (2, 3, 3), v_body = R v_world."""
    rot = np.zeros(18)
    rc = lib().hr_warm_frames(ctypes.byref(inst), _dp(rot))
    if rc != HR_OK:
        raise HrError(rc, "hr_warm_frames failed")
    return rot.reshape(2, 3, 3)


def _fdev(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), ctypes.POINTER(ctypes.c_float))


class MLP:
    """The warm-start network on the device (hand-written CUDA kernels)."""

    NPARAMS = 9347

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        ctx.adopt(self)
        L = lib()
        L.hr_mlp_destroy.restype = None
        p = ctypes.c_void_p()
        ctx._check(L.hr_mlp_create(ctx.p, ctypes.c_ulonglong(seed), ctypes.byref(p)))
        self.p = p

    def close(self):
        if getattr(self, "p", None):
            lib().hr_mlp_destroy(self.p)
            self.p = None

    def __del__(self):
        self.close()

    def set_normalization(self, mean, std, out_scale):
        m = np.ascontiguousarray(mean, np.float32)
        s = np.ascontiguousarray(std, np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self.ctx._check(lib().hr_mlp_set_normalization(self.p, m.ctypes.data_as(fp), s.ctypes.data_as(fp),
                                                       ctypes.c_float(out_scale)))

    def params(self):
        out = np.zeros(self.NPARAMS, np.float32)
        self.ctx._check(lib().hr_mlp_get_params(self.p, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_params(self, p):
        a = np.ascontiguousarray(p, np.float32)
        self.ctx._check(lib().hr_mlp_set_params(self.p, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def train_step(self, X, T, batch, lr, seed=0, random=True, want_loss=False):
        """X, T: torch CUDA float32 tensors (n x 12, n x 3)."""
        loss = ctypes.c_double()
        self.ctx._check(lib().hr_mlp_train_step(self.p, _fdev(X), _fdev(T), ctypes.c_long(X.shape[0]), batch,
                                                1 if random else 0, ctypes.c_ulonglong(seed), ctypes.c_float(lr),
                                                ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def gradient(self, X, T, batch):
        g = np.zeros(self.NPARAMS, np.float32)
        loss = ctypes.c_double()
        self.ctx._check(lib().hr_mlp_gradient(self.p, _fdev(X), _fdev(T), batch,
                                              g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(loss)))
        return loss.value, g

    def infer(self, X, out=None, base=None, raw=None):
        """X: torch CUDA float32 (n x 12); out/base: float64 (3n); raw: float32 (n x 3)."""
        self.ctx._check(lib().hr_mlp_infer(self.p, _fdev(X), ctypes.c_long(X.shape[0]),
                                           None if base is None else _devp(base),
                                           None if out is None else _devp(out),
                                           None if raw is None else _fdev(raw)))

    def infer_frames(self, X, out, base, starts, rot):
        """Body-frame output rotated back: starts (nframes + 1 offsets), rot (nframes, 3, 3)."""
        st = np.ascontiguousarray(starts, np.int64)
        r = np.ascontiguousarray(rot, np.float64).reshape(-1)
        self.ctx._check(lib().hr_mlp_infer_frames(self.p, _fdev(X), ctypes.c_long(X.shape[0]),
                                                  None if base is None else _devp(base), _devp(out),
                                                  len(st) - 1, st.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                                  _dp(r)))

    def save(self, path):
        self.ctx._check(lib().hr_mlp_save(self.p, path.encode()))

    def load(self, path):
        self.ctx._check(lib().hr_mlp_load(self.p, path.encode()))
