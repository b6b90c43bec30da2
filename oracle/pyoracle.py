"""ctypes access to the two oracle libraries (test infrastructure only).

* ``Port``: oracle/liboracle_port.so, the plain-C restatement of the
  reference's BVE and SWE hot path (oracle/bslpm_oracle.c).  Builds from this
  repository alone, so it is the checker on machines without the reference.
* ``Ref``: oracle/_ref/libsbslpm_ref.so, the reference's own src/*.cpp built
  against the shim headers by oracle/Makefile (present where it was built).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module, as the checker or as the timed CPU baseline.  The product
package never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "liboracle_port.so")
REF_PATH = os.path.join(HERE, "_ref", "libsbslpm_ref.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


class OrcPanel(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("id", "top", "left", "bot", "right", "face", "level", "parent")] + [
        ("child", ctypes.c_int * 4),
        ("is_leaf", ctypes.c_int),
    ] + [(n, ctypes.c_double) for n in ("min_xi", "max_xi", "min_eta", "max_eta", "radius", "area")]


class OrcProblem(ctypes.Structure):
    _fields_ = [
        ("levels", ctypes.c_int),
        ("degree", ctypes.c_int),
        ("tracer_count", ctypes.c_int),
        ("mode", ctypes.c_int),
        ("kernel_eps", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("panels", ctypes.POINTER(OrcPanel)),
        ("interp", _D),
        ("x", _D),
        ("y", _D),
        ("z", _D),
        ("area", _D),
        ("n_list", ctypes.c_long),
        ("list", _I),
        ("forcing", ctypes.c_int),
        ("time", ctypes.c_double),
        ("proxy_degree", ctypes.c_int),
        ("leaf_size", ctypes.c_int),
        ("typed", ctypes.c_int),
        ("theta", ctypes.c_double),
    ]


class OrcSweProblem(ctypes.Structure):
    _fields_ = [
        ("levels", ctypes.c_int),
        ("degree", ctypes.c_int),
        ("tracer_count", ctypes.c_int),
        ("kernel_eps", ctypes.c_double),
        ("omega", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("g_over_a", ctypes.c_double),
        ("panels", ctypes.POINTER(OrcPanel)),
        ("interp", _D),
        ("x", _D),
        ("y", _D),
        ("z", _D),
        ("area", _D),
        ("n_list", ctypes.c_long),
        ("list", _I),
        ("map", _I),
        ("counts", _I),
        ("point_count", ctypes.c_int),
        ("base_div", _D),
        ("base_h", _D),
    ]


def panels_to_arrays(panels) -> tuple[np.ndarray, np.ndarray]:
    """(ints P x 13, dbls P x 6) in the column order of ref_get_panels."""
    P = len(panels)
    ints = np.zeros((P, 13), np.int32)
    dbls = np.zeros((P, 6), np.float64)
    for i, p in enumerate(panels):
        ints[i] = [p.id, p.top, p.left, p.bot, p.right, p.face, p.level, p.parent, *p.child, p.is_leaf]
        dbls[i] = [p.min_xi, p.max_xi, p.min_eta, p.max_eta, p.radius, p.area]
    return ints, dbls


class Port:
    """The C restatement.  All arrays are float64 C-contiguous numpy arrays."""

    def __init__(self, path: str = PORT_PATH):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_dual_tree_traversal.restype = ctypes.c_long
        L.orc_dual_tree_traversal.argtypes = [ctypes.c_int, ctypes.POINTER(OrcPanel), ctypes.c_double, _I, ctypes.c_long]
        L.orc_point_locate_panel.restype = ctypes.c_int
        L.orc_point_locate_panel.argtypes = [ctypes.POINTER(OrcPanel), ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.orc_interp_vals_bli.argtypes = [_D] + [ctypes.c_double] * 6 + [ctypes.c_int]
        L.orc_bve_step.argtypes = [ctypes.POINTER(OrcProblem), _D, _D, _D, _D, _D]
        L.orc_interp_to_latlon.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(OrcPanel), _D, ctypes.c_int,
                                           _D, ctypes.c_int, _D, _D]
        L.orc_swe_step.argtypes = [ctypes.POINTER(OrcSweProblem)] + [_D] * 7

    # ---- setup -------------------------------------------------------------
    def build(self, levels: int, degree: int, theta: float | None, exact_cc: bool = False):
        """Panels, interp table, points, areas and (if theta) interaction list."""
        P = 2 * (4**levels - 1)
        A = 6 * 4 ** (levels - 1)
        q = (degree + 1) ** 2
        panels = (OrcPanel * P)()
        self.lib.orc_panels_init(levels, panels)
        interp = np.zeros((q, 4))
        self.lib.orc_interp_init(degree, int(exact_cc), _dp(interp))
        x, y, z, area = (np.zeros((A, q)) for _ in range(4))
        self.lib.orc_spec_points(levels, degree, panels, _dp(interp), _dp(x), _dp(y), _dp(z), _dp(area))
        lst = np.zeros((0, 3), np.int32)
        if theta is not None:
            n = self.lib.orc_dual_tree_traversal(levels, panels, theta, None, 0)
            lst = np.zeros((n, 3), np.int32)
            self.lib.orc_dual_tree_traversal(levels, panels, theta, _ip(lst), n)
        return dict(levels=levels, degree=degree, panels=panels, interp=interp, x=x, y=y, z=z, area=area, list=lst)

    def bli(self, xi, eta, mnx, mxx, mne, mxe, degree):
        out = np.zeros((degree + 1) ** 2)
        self.lib.orc_interp_vals_bli(_dp(out), xi, eta, mnx, mxx, mne, mxe, degree)
        return out

    def locate(self, g, x, y, z) -> int:
        return self.lib.orc_point_locate_panel(g["panels"], x, y, z)

    # ---- passes ------------------------------------------------------------
    def upward_pass(self, g, pots):
        P = len(g["panels"])
        out = np.zeros((P, g["interp"].shape[0]))
        self.lib.orc_upward_pass(g["levels"], g["degree"], g["panels"], _dp(g["interp"]), _dp(g["area"]),
                                 _dp(np.ascontiguousarray(pots)), _dp(out))
        return out

    def downward_pass_3(self, g, t1, t2, t3):
        t1, t2, t3 = (np.array(t, dtype=np.float64, order="C") for t in (t1, t2, t3))
        A, q = g["x"].shape
        s = [np.zeros((A, q)) for _ in range(3)]
        self.lib.orc_downward_pass_3(g["levels"], g["degree"], g["panels"], _dp(g["interp"]), _dp(t1), _dp(t2),
                                     _dp(t3), _dp(s[0]), _dp(s[1]), _dp(s[2]))
        return s

    def vel_interactions(self, g, dx, dy, dz, src, eps):
        P, q = src.shape
        t = [np.zeros((P, q)) for _ in range(3)]
        lst = np.ascontiguousarray(g["list"], dtype=np.int32)
        self.lib.orc_bve_vel_interactions(g["levels"], g["degree"], g["panels"], _dp(g["interp"]),
                                          ctypes.c_long(len(lst)), _ip(lst), _dp(dx), _dp(dy), _dp(dz), _dp(src),
                                          ctypes.c_double(eps), _dp(t[0]), _dp(t[1]), _dp(t[2]))
        return t

    def direct_velocity(self, g, dx, dy, dz, src, eps):
        P, q = src.shape
        t = [np.zeros((P, q)) for _ in range(3)]
        self.lib.orc_bve_direct_velocity(g["levels"], g["degree"], g["panels"], _dp(g["interp"]), _dp(dx), _dp(dy),
                                         _dp(dz), _dp(src), ctypes.c_double(eps), _dp(t[0]), _dp(t[1]), _dp(t[2]))
        return t

    def departure(self, g, v0, v1, v2, v3, dt):
        A, q = g["x"].shape
        dep = [np.zeros((A, q)) for _ in range(3)]
        vs = [np.ascontiguousarray(v, dtype=np.float64) for v in (v0, v1, v2, v3)]
        self.lib.orc_bve_departure(g["levels"], g["degree"], g["panels"], _dp(g["x"]), _dp(g["y"]), _dp(g["z"]),
                                   *[_dp(v) for v in vs], ctypes.c_double(dt), *[_dp(d) for d in dep])
        return dep

    def remap(self, g, dep, vors, tracers, omega):
        A, q = g["x"].shape
        T = 0 if tracers is None else tracers.shape[2]
        tr = np.zeros(1) if tracers is None else np.ascontiguousarray(tracers)
        nv = np.zeros((A, q))
        ntr = np.zeros((A, q, max(T, 1)))
        self.lib.orc_bve_remap(g["levels"], g["degree"], g["panels"], _dp(g["z"]), *[_dp(d) for d in dep],
                               _dp(np.ascontiguousarray(vors)), T, _dp(tr), ctypes.c_double(omega), _dp(nv), _dp(ntr))
        return nv, (ntr if T else None)

    def bve_step(self, g, vors, tracers=None, *, dt, omega, eps, mode=0, nsteps=1, forcing=0, time=0.0,
                 tree=None):
        """nsteps of bve_back_rk4_step from time (forcing 0 none, 1 ssw, 2 ssw2);
        mode 0 the interaction list, 1 direct, 2 treecode with
        tree = (proxy_degree, leaf_size, theta, typed); returns
        (vors, (vx, vy, vz), tracers)."""
        A, q = g["x"].shape
        T = 0 if tracers is None else tracers.shape[2]
        lst = np.ascontiguousarray(g["list"], dtype=np.int32)
        n, leaf, theta, typed = tree if tree is not None else (0, 0, 0.0, 0)
        pb = OrcProblem(g["levels"], g["degree"], T, mode, eps, omega, dt, g["panels"], _dp(g["interp"]), _dp(g["x"]),
                        _dp(g["y"]), _dp(g["z"]), _dp(g["area"]), len(lst), _ip(lst) if len(lst) else None,
                        int(forcing), float(time), int(n), int(leaf), int(typed), float(theta))
        v = np.array(vors, dtype=np.float64, order="C")
        tr = np.zeros(1) if tracers is None else np.array(tracers, dtype=np.float64, order="C")
        vx, vy, vz = (np.zeros((A, q)) for _ in range(3))
        for k in range(nsteps):
            pb.time = float(time) + k * dt
            self.lib.orc_bve_step(ctypes.byref(pb), _dp(v), _dp(vx), _dp(vy), _dp(vz), _dp(tr))
        return v, (vx, vy, vz), (tr if T else None)

    # ---- shallow water v2 --------------------------------------------------
    def swe_vel_interactions(self, g, dx, dy, dz, src_vor, src_div, eps):
        P, q = src_vor.shape
        t = [np.zeros((P, q)) for _ in range(3)]
        lst = np.ascontiguousarray(g["list"], dtype=np.int32)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (dx, dy, dz, src_vor, src_div)]
        self.lib.orc_swe_vel_interactions(g["levels"], g["degree"], g["panels"], _dp(g["interp"]),
                                          ctypes.c_long(len(lst)), _ip(lst), *[_dp(v) for v in a],
                                          ctypes.c_double(eps), _dp(t[0]), _dp(t[1]), _dp(t[2]))
        return t

    def swe_tendencies(self, g, vel, vors, divs, height, surface, omega, g_over_a):
        A, q = g["x"].shape
        out = [np.zeros((A, q)) for _ in range(3)]
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (*vel, vors, divs, height, surface)]
        self.lib.orc_swe_tendencies(g["levels"], g["degree"], g["panels"], _dp(g["x"]), _dp(g["y"]), _dp(g["z"]),
                                    *[_dp(v) for v in a], ctypes.c_double(omega), ctypes.c_double(g_over_a),
                                    *[_dp(o) for o in out])
        return out

    def swe_unify(self, vals, smap, counts):
        v = np.array(vals, dtype=np.float64, order="C")
        m = np.ascontiguousarray(smap, dtype=np.int32)
        c = np.ascontiguousarray(counts, dtype=np.int32)
        self.lib.orc_swe_unify(ctypes.c_int(v.size), _ip(m), _ip(c), ctypes.c_int(c.size), _dp(v))
        return v

    def swe_step(self, g, vors, divs, height, base, smap, counts, tracers=None, *, dt, omega, eps, g_over_a,
                 nsteps=1, driver_unify=False):
        """nsteps of swe_back_rk4_step_2 (base = the three base tendencies);
        driver_unify: the driver's unify of vors, divs and height after each
        step.  Returns (vors, divs, height, (vx, vy, vz), tracers)."""
        A, q = g["x"].shape
        T = 0 if tracers is None else tracers.shape[2]
        lst = np.ascontiguousarray(g["list"], dtype=np.int32)
        m = np.ascontiguousarray(smap, dtype=np.int32)
        c = np.ascontiguousarray(counts, dtype=np.int32)
        bd, bh = (np.ascontiguousarray(b, dtype=np.float64) for b in (base[1], base[2]))
        pb = OrcSweProblem(g["levels"], g["degree"], T, eps, omega, dt, g_over_a, g["panels"], _dp(g["interp"]),
                           _dp(g["x"]), _dp(g["y"]), _dp(g["z"]), _dp(g["area"]), len(lst), _ip(lst), _ip(m),
                           _ip(c), int(c.size), _dp(bd), _dp(bh))
        v, d, h = (np.array(a, dtype=np.float64, order="C") for a in (vors, divs, height))
        tr = np.zeros(1) if tracers is None else np.array(tracers, dtype=np.float64, order="C")
        vel = [np.zeros((A, q)) for _ in range(3)]
        for _ in range(nsteps):
            self.lib.orc_swe_step(ctypes.byref(pb), _dp(v), _dp(d), _dp(h), *[_dp(a) for a in vel], _dp(tr))
            if driver_unify:
                for a in (v, d, h):
                    self.lib.orc_swe_unify(ctypes.c_int(a.size), _ip(m), _ip(c), ctypes.c_int(c.size), _dp(a))
        return v, d, h, tuple(vel), (tr if T else None)

    # ---- treecode (decoupled proxy degree) ---------------------------------
    def bltc_shape(self, levels, degree, leaf_size):
        """(tree levels, particles per tree leaf)."""
        lf, npl = ctypes.c_int(), ctypes.c_int()
        self.lib.orc_bltc_shape(levels, degree, leaf_size, ctypes.byref(lf), ctypes.byref(npl))
        return lf.value, npl.value

    def bltc_list(self, levels, degree, leaf_size, n, theta):
        f = self.lib.orc_bltc_list
        f.restype = ctypes.c_long
        cnt = f(levels, degree, leaf_size, n, ctypes.c_double(theta), None, ctypes.c_long(0))
        out = np.zeros((cnt, 3), np.int32)
        f(levels, degree, leaf_size, n, ctypes.c_double(theta), _ip(out), ctypes.c_long(cnt))
        return out

    def bltc_upward(self, levels, degree, leaf_size, n, sx, sy, sz, w):
        lf, _ = self.bltc_shape(levels, degree, leaf_size)
        P = 2 * (4**lf - 1)
        out = np.zeros((P, (n + 1) ** 2))
        a = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in (sx, sy, sz, w)]
        self.lib.orc_bltc_upward(levels, degree, leaf_size, n, *[_dp(v) for v in a], _dp(out))
        return out

    def bltc_downward(self, levels, degree, leaf_size, n, T, tx, ty, tz):
        """(proxy targets after the parent-to-child passes, 3 x N particle values)."""
        t = np.array(T, dtype=np.float64, order="C")
        a = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in (tx, ty, tz)]
        u = np.zeros((3, a[0].size))
        self.lib.orc_bltc_downward(levels, degree, leaf_size, n, _dp(t), *[_dp(v) for v in a], _dp(u))
        return t, u

    def bltc_velocity_swe(self, levels, degree, leaf_size, n, theta, eps, typed, t, s, w, d, wd):
        """Shallow-water treecode velocity (3 x N): vorticity sources s (strengths w), divergence
        sources d (strengths wd)."""
        a = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in (*t, *s, w, *d, wd)]
        u = np.zeros((3, a[0].size))
        self.lib.orc_bltc_velocity_swe(levels, degree, leaf_size, n, ctypes.c_double(theta), ctypes.c_double(eps),
                                       int(typed), *[_dp(v) for v in a], _dp(u))
        return u

    def bltc_velocity(self, levels, degree, leaf_size, n, theta, eps, typed, t, s, w):
        """Treecode velocity (3 x N) at targets t = (x, y, z) of sources s with strengths w."""
        a = [np.ascontiguousarray(v, dtype=np.float64).ravel() for v in (*t, *s, w)]
        u = np.zeros((3, a[0].size))
        self.lib.orc_bltc_velocity(levels, degree, leaf_size, n, ctypes.c_double(theta), ctypes.c_double(eps),
                                   int(typed), *[_dp(v) for v in a], _dp(u))
        return u

    def poisson_fmm_interactions(self, g, source, target):
        """poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34): target += ..."""
        t = np.ascontiguousarray(target, float).copy()
        lst = np.ascontiguousarray(g["list"], np.int32)
        self.lib.orc_poisson_fmm_interactions(g["levels"], g["degree"], g["panels"], _dp(g["interp"]),
                                              ctypes.c_long(len(lst)), _ip(lst),
                                              _dp(np.ascontiguousarray(source, float)), _dp(t))
        return t

    def downward_pass(self, g, target):
        """downward_pass (src/fmm_funcs.cpp:357-372): (updated proxy targets, leaf values)."""
        t = np.ascontiguousarray(target, float).copy()
        s = np.zeros_like(g["x"])
        self.lib.orc_downward_pass(g["levels"], g["degree"], g["panels"], _dp(g["interp"]), _dp(t), _dp(s))
        return t, s

    def interp_to_latlon(self, g, data, lats, lons):
        """interp_to_latlon_host (src/interp_funcs.hpp:22-77): [nlat][nlon]."""
        lats, lons = np.ascontiguousarray(lats, float), np.ascontiguousarray(lons, float)
        out = np.zeros((len(lats), len(lons)))
        self.lib.orc_interp_to_latlon(g["levels"], g["degree"], g["panels"], _dp(np.ascontiguousarray(data)),
                                      len(lats), _dp(lats), len(lons), _dp(lons), _dp(out))
        return out

    def xyz_vel_to_uv_vel(self, x, y, z, vx, vy, vz):
        """xyz_vel_to_uv_vel (src/general_utils_impl.hpp:195-229): (u, v)."""
        a = [np.ascontiguousarray(t, float).ravel() for t in (x, y, z, vx, vy, vz)]
        u, v = np.zeros(a[0].size), np.zeros(a[0].size)
        self.lib.orc_xyz_vel_to_uv_vel(ctypes.c_long(a[0].size), *[_dp(t) for t in a], _dp(u), _dp(v))
        return u.reshape(np.shape(x)), v.reshape(np.shape(x))

    def direct_sum_inv_lap(self, x, y, z, area, pots):
        n = len(x)
        out = np.zeros(n)
        self.lib.orc_direct_sum_inv_lap(n, _dp(x), _dp(y), _dp(z), _dp(area), _dp(pots), _dp(out))
        return out


class Ref:
    """The reference's own code (oracle/_ref/libsbslpm_ref.so)."""

    def __init__(self, path: str = REF_PATH):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int]
        for name in ("ref_destroy", "ref_sizes", "ref_get_panels", "ref_get_interactions", "ref_get_points",
                     "ref_bve_initialize", "ref_bve_step", "ref_bve_vel_interactions", "ref_upward_pass",
                     "ref_downward_pass_3", "ref_bve_departure", "ref_bve_remap", "ref_set_area"):
            getattr(L, name).restype = None
        L.ref_bve_step.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int]
        L.ref_bve_departure.argtypes = [ctypes.c_void_p, _D, _D, _D, _D, ctypes.c_double, _D, _D, _D]
        L.ref_point_locate_panel.restype = ctypes.c_int
        L.ref_point_locate_panel.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_interp_vals_bli.argtypes = [_D] + [ctypes.c_double] * 6 + [ctypes.c_int]
        L.ref_num_threads.restype = ctypes.c_int
        L.ref_swe_map.restype = ctypes.c_int
        L.ref_interp_to_latlon.restype = None
        L.ref_interp_to_latlon.argtypes = [ctypes.c_void_p, _D, ctypes.c_int, _D, ctypes.c_int, _D, _D]
        L.ref_xyz_vel_to_uv_vel.restype = None
        L.ref_poisson_fmm.restype = None
        L.ref_set_forcing.restype = None
        L.ref_poisson_fmm_interactions.restype = None
        for name in ("ref_unify", "ref_swe_vel_interactions", "ref_swe_tendency", "ref_swe_init", "ref_swe_step"):
            getattr(L, name).restype = None
        L.ref_swe_step.argtypes = [ctypes.c_void_p] + [_D] * 10 + [_I, _I, ctypes.c_double, ctypes.c_int,
                                                                   ctypes.c_int]

    def create(self, levels, degree, theta, eps, omega, delta_t, tracer_count):
        h = ctypes.c_void_p(self.lib.ref_create(levels, degree, theta, eps, omega, delta_t, tracer_count))
        sz = np.zeros(5, np.int32)
        self.lib.ref_sizes(h, _ip(sz))
        P, A, q, I, _ = (int(v) for v in sz)
        return dict(h=h, P=P, A=A, q=q, I=I, T=tracer_count, levels=levels, degree=degree)

    def destroy(self, c):
        self.lib.ref_destroy(c["h"])

    def set_area(self, c, area):
        """Replaces the quadrature weights (A x q) the later calls read."""
        self.lib.ref_set_area(c["h"], _dp(np.ascontiguousarray(area, dtype=np.float64)))

    def panels(self, c):
        ints = np.zeros((c["P"], 13), np.int32)
        dbls = np.zeros((c["P"], 6))
        self.lib.ref_get_panels(c["h"], _ip(ints), _dp(dbls))
        return ints, dbls

    def interactions(self, c):
        out = np.zeros((c["I"], 3), np.int32)
        self.lib.ref_get_interactions(c["h"], _ip(out))
        return out

    def points(self, c):
        A, q = c["A"], c["q"]
        x, y, z, area = (np.zeros((A, q)) for _ in range(4))
        interp = np.zeros((q, 4))
        self.lib.ref_get_points(c["h"], _dp(x), _dp(y), _dp(z), _dp(area), _dp(interp))
        return x, y, z, area, interp

    def initialize(self, c, ic: str, balance: bool):
        v = np.zeros((c["A"], c["q"]))
        self.lib.ref_bve_initialize(c["h"], ic.encode(), int(balance), _dp(v))
        return v

    def bve_step(self, c, vors, tracers=None, time=0.0, nsteps=1):
        A, q, T = c["A"], c["q"], c["T"]
        v = np.array(vors, dtype=np.float64, order="C")
        tr = np.zeros((A, q, max(T, 1))) if tracers is None else np.array(tracers, dtype=np.float64, order="C")
        vx, vy, vz = (np.zeros((A, q)) for _ in range(3))
        self.lib.ref_bve_step(c["h"], _dp(v), _dp(vx), _dp(vy), _dp(vz), _dp(tr), time, nsteps)
        return v, (vx, vy, vz), (tr if T else None)

    def vel_interactions(self, c, dx, dy, dz, src):
        t = [np.zeros((c["P"], c["q"])) for _ in range(3)]
        self.lib.ref_bve_vel_interactions(c["h"], _dp(dx), _dp(dy), _dp(dz), _dp(src), _dp(t[0]), _dp(t[1]), _dp(t[2]))
        return t

    def upward_pass(self, c, pots):
        out = np.zeros((c["P"], c["q"]))
        self.lib.ref_upward_pass(c["h"], _dp(np.ascontiguousarray(pots)), _dp(out))
        return out

    def downward_pass_3(self, c, t1, t2, t3):
        t1, t2, t3 = (np.array(t, dtype=np.float64, order="C") for t in (t1, t2, t3))
        s = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        self.lib.ref_downward_pass_3(c["h"], _dp(t1), _dp(t2), _dp(t3), _dp(s[0]), _dp(s[1]), _dp(s[2]))
        return s

    def departure(self, c, v0, v1, v2, v3, dt):
        dep = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        vs = [np.ascontiguousarray(v, dtype=np.float64) for v in (v0, v1, v2, v3)]
        self.lib.ref_bve_departure(c["h"], *[_dp(v) for v in vs], dt, *[_dp(d) for d in dep])
        return dep

    def remap(self, c, dep, vors, tracers):
        A, q, T = c["A"], c["q"], c["T"]
        tr = np.zeros((A, q, max(T, 1))) if tracers is None else np.ascontiguousarray(tracers)
        nv = np.zeros((A, q))
        ntr = np.zeros((A, q, max(T, 1)))
        self.lib.ref_bve_remap(c["h"], *[_dp(d) for d in dep], _dp(np.ascontiguousarray(vors)), _dp(tr), _dp(nv), _dp(ntr))
        return nv, (ntr if T else None)

    def bli(self, xi, eta, mnx, mxx, mne, mxe, degree):
        out = np.zeros((degree + 1) ** 2)
        self.lib.ref_interp_vals_bli(_dp(out), xi, eta, mnx, mxx, mne, mxe, degree)
        return out

    def locate(self, c, x, y, z) -> int:
        return self.lib.ref_point_locate_panel(c["h"], x, y, z)

    def set_forcing(self, c, forcing: int):
        """forcing 0 none, 1 ssw, 2 ssw2 (RunConfig::forcing / forcing_type)."""
        self.lib.ref_set_forcing(c["h"], int(forcing))

    def poisson_fmm(self, c, pots):
        """The Poisson FMM driver's solve: (proxy source, proxy target, soln)."""
        P, A, q = c["P"], c["A"], c["q"]
        src, tgt, soln = np.zeros((P, q)), np.zeros((P, q)), np.zeros((A, q))
        self.lib.ref_poisson_fmm(c["h"], _dp(np.ascontiguousarray(pots, float)), _dp(src), _dp(tgt), _dp(soln))
        return src, tgt, soln

    def poisson_fmm_interactions(self, c, source, target):
        t = np.ascontiguousarray(target, float).copy()
        self.lib.ref_poisson_fmm_interactions(c["h"], _dp(np.ascontiguousarray(source, float)), _dp(t))
        return t

    def interp_to_latlon(self, c, data, lats, lons):
        lats, lons = np.ascontiguousarray(lats, float), np.ascontiguousarray(lons, float)
        out = np.zeros((len(lats), len(lons)))
        self.lib.ref_interp_to_latlon(c["h"], _dp(np.ascontiguousarray(data)), len(lats), _dp(lats), len(lons),
                                      _dp(lons), _dp(out))
        return out

    def xyz_vel_to_uv_vel(self, c, vx, vy, vz):
        u, v = np.zeros(np.shape(vx)), np.zeros(np.shape(vx))
        self.lib.ref_xyz_vel_to_uv_vel(c["h"], *[_dp(np.ascontiguousarray(t)) for t in (vx, vy, vz)], _dp(u), _dp(v))
        return u, v

    def direct_sum_inv_lap(self, x, y, z, area, pots):
        n = len(x)
        out = np.zeros(n)
        self.lib.ref_direct_sum_inv_lap(n, _dp(x), _dp(y), _dp(z), _dp(area), _dp(pots), _dp(out))
        return out

    # ---- shallow water (SWE v2) -------------------------------------------

    # ---- the irregular-point ("_ll") FMM on the particle grid's truncated tree ----
    def ll_create(self, levels, degree, leaf_size, proxy_degree, theta, eps):
        L = self.lib
        L.ref_ll_create.restype = ctypes.c_void_p
        L.ref_ll_create.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double]
        for name in ("ref_ll_destroy", "ref_ll_sizes", "ref_ll_list", "ref_ll_upward", "ref_ll_downward",
                     "ref_ll_velocity"):
            getattr(L, name).restype = None
        h = ctypes.c_void_p(L.ref_ll_create(levels, degree, leaf_size, proxy_degree, theta, eps))
        sz = np.zeros(5, np.int32)
        L.ref_ll_sizes(h, _ip(sz))
        Pf, Lf, npl, qx, I = (int(v) for v in sz)
        A, q = 6 * 4 ** (levels - 1), (degree + 1) ** 2
        return dict(h=h, Pf=Pf, Lf=Lf, npl=npl, qx=qx, I=I, A=A, q=q)

    def ll_destroy(self, c):
        self.lib.ref_ll_destroy(c["h"])

    def ll_list(self, c):
        out = np.zeros((c["I"], 3), np.int32)
        self.lib.ref_ll_list(c["h"], _ip(out))
        return out

    def ll_upward(self, c, pots):
        out = np.zeros((c["Pf"], c["qx"]))
        self.lib.ref_ll_upward(c["h"], _dp(np.ascontiguousarray(pots, dtype=np.float64)), _dp(out))
        return out

    def ll_downward(self, c, t1, t2, t3):
        t = [np.ascontiguousarray(v, dtype=np.float64) for v in (t1, t2, t3)]
        s = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        self.lib.ref_ll_downward(c["h"], *[_dp(v) for v in t], *[_dp(v) for v in s])
        return s

    def ll_velocity(self, c, vors, divs=None):
        out = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        d = None if divs is None else _dp(np.ascontiguousarray(divs, dtype=np.float64))
        self.lib.ref_ll_velocity(c["h"], _dp(np.ascontiguousarray(vors, dtype=np.float64)), d, *[_dp(v) for v in out])
        return out

    def swe_map(self, c):
        """cubed_sphere_2d_to_1d: (two_d_to_1d A x q int32, counts U int32)."""
        U = c["A"] * c["degree"] ** 2 + 2
        m = np.zeros((c["A"], c["q"]), np.int32)
        n = np.zeros(U, np.int32)
        u = self.lib.ref_swe_map(c["h"], _ip(m), _ip(n))
        assert u == U
        return m, n

    def unify(self, c, vals, smap):
        v = np.array(vals, dtype=np.float64, order="C")
        self.lib.ref_unify(c["h"], _dp(v), _ip(smap[0]), _ip(smap[1]))
        return v

    def swe_vel_interactions(self, c, dx, dy, dz, src_vor, src_div):
        t = [np.zeros((c["P"], c["q"])) for _ in range(3)]
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (dx, dy, dz, src_vor, src_div)]
        self.lib.ref_swe_vel_interactions(c["h"], *[_dp(v) for v in a], *[_dp(v) for v in t])
        return t

    def swe_tendency(self, c, vel, vors, divs, height, surface):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (*vel, vors, divs, height, surface)]
        out = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        self.lib.ref_swe_tendency(c["h"], *[_dp(v) for v in a], *[_dp(v) for v in out])
        return out

    def swe_init(self, c, vors, divs, height, smap):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (vors, divs, height)]
        vel = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        base = [np.zeros((c["A"], c["q"])) for _ in range(3)]
        self.lib.ref_swe_init(c["h"], *[_dp(v) for v in a], *[_dp(v) for v in vel], *[_dp(v) for v in base],
                              _ip(smap[0]), _ip(smap[1]))
        return vel, base

    def swe_step(self, c, vors, divs, height, base, smap, vel=None, tracers=None, time=0.0, nsteps=1,
                 driver_unify=False):
        A, q, T = c["A"], c["q"], c["T"]
        v, d, h = (np.array(a, dtype=np.float64, order="C") for a in (vors, divs, height))
        vel = [np.zeros((A, q)) for _ in range(3)] if vel is None else [np.array(a, dtype=np.float64, order="C")
                                                                        for a in vel]
        tr = np.zeros((A, q, max(T, 1))) if tracers is None else np.array(tracers, dtype=np.float64, order="C")
        b = [np.ascontiguousarray(a, dtype=np.float64) for a in base]
        self.lib.ref_swe_step(c["h"], _dp(v), _dp(d), _dp(h), *[_dp(a) for a in vel], _dp(tr),
                              *[_dp(a) for a in b], _ip(smap[0]), _ip(smap[1]), time, nsteps, int(driver_unify))
        return v, d, h, vel, (tr if T else None)
