"""ctypes wrappers of the checkers (TEST INFRASTRUCTURE ONLY).

* `Ref`    -- the reference's own CPU build (oracle/_ref/libcryoref*.so).
* `Oracle` -- the plain-C restatement (oracle/libcryo_oracle.so).

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
Both expose the same small surface (set_particles, step, relax, field, ...)
so a test can run the same scenario through either.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import ref_abi as cabi  # noqa: E402  (struct layouts of include/cryosph_b200.h; nothing from the package)

REF_LIB = os.path.join(HERE, "_ref", "libcryoref.so")
REF_LIB64 = os.path.join(HERE, "_ref", "libcryoref64.so")
REF_LIB_CUDA = os.path.join(HERE, "_ref", "libcryoref_cuda.so")  # make refcuda: the reference's CUDA backend
ORACLE_LIB = os.path.join(HERE, "libcryo_oracle.so")

# geometry node kinds (ref_driver.h)
CYLINDER, CAPSULE, SPHERE, BOX, TRANSLATED, DIFFERENCE, UNION = range(7)


class GeomNode(C.Structure):
    _fields_ = [("kind", C.c_int), ("a", C.c_int), ("b", C.c_int), ("p", C.c_double * 3)]


class Fill(C.Structure):
    _fields_ = [("mode", C.c_int), ("fill_fraction", C.c_double), ("settle_direction", C.c_float * 3),
                ("bubble_center", C.c_float * 3), ("include_vapor", C.c_int), ("wall_layers", C.c_int),
                ("T_liquid", C.c_float), ("T_vapor", C.c_float), ("T_wall", C.c_float),
                ("heater_zmin", C.c_double), ("heater_zmax", C.c_double)]


def make_fill(mode=0, fill_fraction=0.5, settle=(0, 0, -1), bubble=(0, 0, 0), include_vapor=True, wall_layers=3,
              T_liquid=float("nan"), T_vapor=float("nan"), T_wall=float("nan"), heater_zmin=-np.inf,
              heater_zmax=np.inf):
    f = Fill()
    f.mode = mode
    f.fill_fraction = fill_fraction
    f.settle_direction[:] = list(settle)
    f.bubble_center[:] = list(bubble)
    f.include_vapor = int(include_vapor)
    f.wall_layers = wall_layers
    f.T_liquid, f.T_vapor, f.T_wall = T_liquid, T_vapor, T_wall
    f.heater_zmin, f.heater_zmax = heater_zmin, heater_zmax
    return f


def geom(nodes):
    """nodes: list of (kind, a, b, (p0, p1, p2)); the last is the root."""
    arr = (GeomNode * len(nodes))()
    for k, (kind, a, b, p) in enumerate(nodes):
        arr[k].kind, arr[k].a, arr[k].b = kind, a, b
        pp = list(p) + [0.0] * (3 - len(p))
        arr[k].p[:] = pp
    return arr


def _declare(L, has_tank):
    vp, i, f, d = C.c_void_p, C.c_int, C.c_float, C.c_double
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    sig = {
        "create": (vp, [C.POINTER(cabi.Config), C.POINTER(cabi.Fluid), C.c_char_p, i]),
        "destroy": (None, [vp]),
        "last_error": (C.c_char_p, [vp]),
        "set_particles": (i, [vp, C.POINTER(cabi.HostParticles), fp, fp]),
        "step": (i, [vp, C.c_longlong]),
        "run_until": (i, [vp, d]),
        "relax": (i, [vp, d, f]),
        "next_dt": (i, [vp, dp]),
        "time": (i, [vp, dp, C.POINTER(C.c_longlong), dp]),
        "num_particles": (i, [vp]),
        "diagnostics": (i, [vp, C.POINTER(cabi.Diagnostics)]),
        "get_field": (i, [vp, i, vp]),
        "set_gravity": (i, [vp, fp]),
        "set_frame_motion": (i, [vp, fp, fp, fp, fp]),
        "set_maneuver": (i, [vp, i, dp, fp, fp, fp]),
        "clear_frame_motion": (i, [vp]),
        "set_heater_power": (i, [vp, f]),
        "set_contact_angle": (i, [vp, f]),
        "damp_velocities": (i, [vp, f]),
        "probe_pressure": (i, [vp, fp, i, fp]),
        "pass": (i, [vp, i]),
        "set_dt": (i, [vp, f]),
        "neighbor_lists": (i, [vp, vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "grid_info": (i, [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), C.POINTER(i), fp, fp]),
        "grid_tables": (i, [vp, vp, vp]),
        "params": (i, [vp, fp, fp, fp, fp, fp, fp, fp]),
        "real_size": (i, []),
        "set_threads": (None, [i]),
        "get_threads": (i, []),
    }
    if has_tank:
        sig.update({
            "build_tank": (i, [vp, C.POINTER(GeomNode), i, C.POINTER(Fill)]),
            "tank_particles": (i, [C.POINTER(GeomNode), i, C.POINTER(cabi.Fluid), f, C.POINTER(Fill),
                                   C.POINTER(cabi.HostOut)]),
            "free_particles": (None, [C.POINTER(cabi.HostOut)]),
            "tank_domain": (i, [C.POINTER(GeomNode), i, f, i, fp, fp]),
            "geom_sdf": (d, [C.POINTER(GeomNode), i, d, d, d]),
            "neighbor_stats": (i, [vp, f, vp, vp]),
        })
    return sig


class _Checker:
    prefix = ""
    has_tank = False

    def __init__(self, path, cfg: "cabi.Config", fluid: "cabi.Fluid"):
        self.L = C.CDLL(path)
        for name, (res, args) in _declare(self.L, self.has_tank).items():
            fn = getattr(self.L, self.prefix + name)
            fn.restype, fn.argtypes = res, args
        err = C.create_string_buffer(512)
        cfg, fluid = cabi.as_struct(cabi.Config, cfg), cabi.as_struct(cabi.Fluid, fluid)
        self.h = self._f("create")(C.byref(cfg), C.byref(fluid), err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        self.real = np.float64 if self._f("real_size")() == 8 else np.float32

    def _f(self, name):
        return getattr(self.L, self.prefix + name)

    def close(self):
        if getattr(self, "h", None):
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc:
            raise cabi.RefError(rc, self._f("last_error")(self.h).decode())

    def set_threads(self, n):
        self._f("set_threads")(int(n))

    def set_particles(self, arrays, lo, hi):
        keep = []
        hp = cabi.host_particles(arrays, keep)
        self.check(self._f("set_particles")(self.h, C.byref(hp), cabi.vec3(lo), cabi.vec3(hi)))

    def step(self, n=1):
        self.check(self._f("step")(self.h, int(n)))

    def run_until(self, t):
        self.check(self._f("run_until")(self.h, float(t)))

    def relax(self, duration, damping=0.98):
        self.check(self._f("relax")(self.h, float(duration), float(damping)))

    def next_dt(self):
        d = C.c_double()
        self.check(self._f("next_dt")(self.h, C.byref(d)))
        return d.value

    def time(self):
        t, s, dt = C.c_double(), C.c_longlong(), C.c_double()
        self.check(self._f("time")(self.h, C.byref(t), C.byref(s), C.byref(dt)))
        return t.value, s.value, dt.value

    def num_particles(self):
        return self._f("num_particles")(self.h)

    def diagnostics(self):
        d = cabi.Diagnostics()
        self.check(self._f("diagnostics")(self.h, C.byref(d)))
        return d

    def field(self, name):
        n = self.num_particles()
        out = np.empty(cabi.field_shape(name, n), dtype=cabi.field_dtype(name, self.real))
        self.check(self._f("get_field")(self.h, cabi.FIELD_ID[name], out.ctypes.data_as(C.c_void_p)))
        return out

    def run_pass(self, name):
        self.check(self._f("pass")(self.h, cabi.PASS_ID[name]))

    def set_pass_dt(self, dt):
        self.check(self._f("set_dt")(self.h, float(dt)))

    def set_gravity(self, g):
        self.check(self._f("set_gravity")(self.h, cabi.vec3(g)))

    def set_frame_motion(self, a=(0, 0, 0), w=(0, 0, 0), wd=(0, 0, 0), o=(0, 0, 0)):
        self.check(self._f("set_frame_motion")(self.h, cabi.vec3(a), cabi.vec3(w), cabi.vec3(wd), cabi.vec3(o)))

    def set_maneuver(self, times, acc, omega=None, origin=(0, 0, 0)):
        t = np.ascontiguousarray(times, np.float64)
        a = np.ascontiguousarray(acc, np.float32)
        w = None if omega is None else np.ascontiguousarray(omega, np.float32)
        self.check(self._f("set_maneuver")(self.h, len(t), t.ctypes.data_as(C.POINTER(C.c_double)),
                                           a.ctypes.data_as(C.POINTER(C.c_float)),
                                           None if w is None else w.ctypes.data_as(C.POINTER(C.c_float)),
                                           cabi.vec3(origin)))

    def set_heater_power(self, w):
        self.check(self._f("set_heater_power")(self.h, float(w)))

    def set_contact_angle(self, deg):
        self.check(self._f("set_contact_angle")(self.h, float(deg)))

    def damp_velocities(self, f):
        self.check(self._f("damp_velocities")(self.h, float(f)))

    def probe_pressure(self, pts):
        pts = np.ascontiguousarray(pts, np.float32)
        out = np.empty(len(pts), np.float32)
        self.check(self._f("probe_pressure")(self.h, pts.ctypes.data_as(C.POINTER(C.c_float)), len(pts),
                                             out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def neighbor_lists(self):
        n = self.num_particles()
        counts = np.empty(n, np.int32)
        total = C.c_longlong()
        self.check(self._f("neighbor_lists")(self.h, counts.ctypes.data_as(C.c_void_p), None, 0, C.byref(total)))
        lst = np.empty(max(total.value, 1), np.int32)
        self.check(self._f("neighbor_lists")(self.h, counts.ctypes.data_as(C.c_void_p),
                                             lst.ctypes.data_as(C.c_void_p), total.value, C.byref(total)))
        return counts, lst[: total.value]

    def grid_info(self):
        nc, nx, ny, nz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        o, ic = (C.c_float * 3)(), C.c_float()
        self.check(self._f("grid_info")(self.h, C.byref(nc), C.byref(nx), C.byref(ny), C.byref(nz), o,
                                        C.byref(ic)))
        return dict(num_cells=nc.value, nx=nx.value, ny=ny.value, nz=nz.value, origin=tuple(o), inv_cell=ic.value)

    def cell_tables(self):
        nc = self.grid_info()["num_cells"]
        cs, ce = np.empty(nc, np.int32), np.empty(nc, np.int32)
        self.check(self._f("grid_tables")(self.h, cs.ctypes.data_as(C.c_void_p), ce.ctypes.data_as(C.c_void_p)))
        return cs, ce

    def params(self):
        vals = [C.c_float() for _ in range(7)]
        self.check(self._f("params")(self.h, *[C.byref(v) for v in vals]))
        keys = ["c0", "h", "vol0", "support2", "T_sat", "dt", "heat_inv_norm"]
        return {k: v.value for k, v in zip(keys, vals)}


class Ref(_Checker):
    """The reference's own CPU implementation (FP32 by default, FP64 with fp64=True)."""
    prefix = "ref_"
    has_tank = True

    def __init__(self, cfg, fluid, fp64=False, cuda=False):
        super().__init__(REF_LIB_CUDA if cuda else (REF_LIB64 if fp64 else REF_LIB), cfg, fluid)

    def build_tank(self, nodes, fill):
        g = geom(nodes)
        self.check(self._f("build_tank")(self.h, g, len(nodes), C.byref(fill)))

    def neighbor_stats(self, radius):
        n = self.num_particles()
        c = np.empty(n, np.int32)
        s = np.empty(n, np.uint64)
        self.check(self._f("neighbor_stats")(self.h, float(radius), c.ctypes.data_as(C.c_void_p),
                                             s.ctypes.data_as(C.c_void_p)))
        return c, s


def ref_available(fp64=False, cuda=False):
    return os.path.exists(REF_LIB_CUDA if cuda else (REF_LIB64 if fp64 else REF_LIB))


def oracle_available():
    return os.path.exists(ORACLE_LIB)


def _ref_lib_for_tools():
    L = C.CDLL(REF_LIB)
    for name, (res, args) in _declare(L, True).items():
        fn = getattr(L, "ref_" + name)
        fn.restype, fn.argtypes = res, args
    return L


def tank_particles(nodes, fluid, dx, fill):
    """The reference's lattice generator (geometry.cpp:242-330) as numpy arrays."""
    L = _ref_lib_for_tools()
    g = geom(nodes)
    out = cabi.HostOut()
    fluid = cabi.as_struct(cabi.Fluid, fluid)
    rc = L.ref_tank_particles(g, len(nodes), C.byref(fluid), float(dx), C.byref(fill), C.byref(out))
    if rc:
        raise cabi.RefError(rc, "tank_particles failed")
    n = out.n
    res = {
        "x": np.ctypeslib.as_array(out.x, (n, 3)).copy(),
        "v": np.ctypeslib.as_array(out.v, (n, 3)).copy(),
        "nrm": np.ctypeslib.as_array(out.nrm, (n, 3)).copy(),
        "m": np.ctypeslib.as_array(out.m, (n,)).copy(),
        "rho": np.ctypeslib.as_array(out.rho, (n,)).copy(),
        "T": np.ctypeslib.as_array(out.T, (n,)).copy(),
        "phase": np.ctypeslib.as_array(out.phase, (n,)).copy(),
        "flags": np.ctypeslib.as_array(out.flags, (n,)).copy(),
        "id": np.ctypeslib.as_array(out.id, (n,)).copy(),
    }
    L.ref_free_particles(C.byref(out))
    return res


def tank_domain(nodes, dx, wall_layers=3):
    L = _ref_lib_for_tools()
    g = geom(nodes)
    lo, hi = (C.c_float * 3)(), (C.c_float * 3)()
    rc = L.ref_tank_domain(g, len(nodes), float(dx), wall_layers, lo, hi)
    if rc:
        raise cabi.RefError(rc, "tank_domain failed")
    return tuple(lo), tuple(hi)


class Oracle(_Checker):
    """The plain-C restatement of the hot path (cryo_oracle.c)."""
    prefix = "orc_"
    has_tank = False

    def __init__(self, cfg, fluid):
        super().__init__(ORACLE_LIB, cfg, fluid)
        self.L.orc_set_field.restype = C.c_int
        self.L.orc_set_field.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        self.L.orc_grid_sort.restype = C.c_int
        self.L.orc_grid_sort.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        self.L.orc_scalars.restype = C.c_int
        self.L.orc_scalars.argtypes = [C.c_void_p, C.POINTER(C.c_double)]

    def set_field(self, name, data):
        n = self.num_particles()
        a = np.ascontiguousarray(data, dtype=cabi.field_dtype(name, self.real)).reshape(cabi.field_shape(name, n))
        self.check(self.L.orc_set_field(self.h, cabi.FIELD_ID[name], a.ctypes.data_as(C.c_void_p)))

    def grid_sort(self):
        n = self.num_particles()
        k = np.empty(n, np.uint32)
        p = np.empty(n, np.uint32)
        self.check(self.L.orc_grid_sort(self.h, k.ctypes.data_as(C.c_void_p), p.ctypes.data_as(C.c_void_p)))
        return k, p

    def scalars(self):
        out = (C.c_double * 8)()
        self.check(self.L.orc_scalars(self.h, out))
        keys = ["p_ullage", "fluid_volume0", "v_max", "a_max", "Tv_max", "spacing_ratio", "nu_t_max", "heat_input"]
        return dict(zip(keys, list(out)))
