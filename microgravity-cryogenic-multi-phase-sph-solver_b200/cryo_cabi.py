"""ctypes view of the C ABI declared in include/cryosph_b200.h.

`load()` opens libcryosph_b200.so (built in-tree by build.py) and declares the
argument types of every entry point.  The struct classes mirror the C structs
field for field; `config_default()`, `fluid_preset()` fill them from the
library.  Errors come back as CryoError carrying the status code and message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libcryosph_b200.so"

# status codes
CRYO_OK, CRYO_EINVAL, CRYO_ERANGE, CRYO_ERUNTIME, CRYO_ECUDA, CRYO_EDEVICE = range(6)
CRYO_ARITH_EXACT, CRYO_ARITH_FAST = 0, 1
# phases / flags
LIQUID, VAPOR, WALL, DEAD = 0, 1, 2, 3
FLAG_HEATED, FLAG_SOURCE, FLAG_TARGET_VAPOR, FLAG_DYING = 1, 2, 4, 8
FLUID_CUSTOM, FLUID_LH2, FLUID_LN2, FLUID_LOX, FLUID_LCH4, FLUID_H2O = range(6)

FIELDS = [
    "x", "v", "vt", "nrm", "m", "m0", "rho", "T", "phase", "flags", "id",
    "a", "ab", "fw", "mw", "ns", "vw",
    "p", "drho", "dTdt", "sigma", "kappa", "nu_t", "alpha",
    "wall_w", "heat_w", "out_m", "out_h", "w_norm", "rmin", "p_wv",
]
FIELD_ID = {name: k for k, name in enumerate(FIELDS)}
VEC_FIELDS = {"x", "v", "vt", "nrm", "a", "ab", "fw", "mw", "ns", "vw"}
U8_FIELDS = {"phase", "flags"}
U32_FIELDS = {"id"}

PASSES = [
    "kick_drift", "grid_build", "density", "normalize_masses", "eos", "wall_boundary", "interface",
    "transport", "sps", "momentum", "smooth_normals", "csf", "akinci", "density_rate", "thermal",
    "maxima", "kick", "shifting", "pc_sources", "pc_normalize", "pc_apply", "rebalance", "split",
    "venting", "saturation",
]
PASS_ID = {name: k for k, name in enumerate(PASSES)}


class Fluid(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "rho_liquid", "rho_vapor", "mu_liquid", "mu_vapor", "k_liquid", "k_vapor",
        "cp_liquid", "cp_vapor", "sigma", "h_fg", "T_sat", "p_sat", "R_gas")]


_F, _I = C.c_float, C.c_int
CONFIG_FIELDS = [
    ("dx", _F), ("h_factor", _F), ("kernel", _I), ("density_mode", _I), ("normalize_initial_masses", _I),
    ("gravity", _F * 3), ("velocity_scale", _F), ("sound_speed", _F), ("tait_gamma", _F),
    ("background_pressure", _F), ("vapor_stiffness", _F), ("clamp_negative_pressure", _I),
    ("transport_velocity", _I), ("transport_background_factor", _F), ("transport_stress", _I),
    ("transport_interface_only", _I), ("particle_shifting", _I), ("shifting_strength", _F),
    ("artificial_viscosity", _F), ("artificial_viscosity_vapor", _F), ("delta_sph", _F),
    ("no_slip", _I), ("sps_turbulence", _I), ("smagorinsky_cs", _F),
    ("surface_tension", _I), ("contact_angle_deg", _F), ("contact_angle_wall_weight", _F),
    ("wall_colour", _I), ("wetting_model", _I), ("csf_smooth_normals", _I), ("csf_balanced", _I),
    ("akinci_gamma", _F), ("akinci_beta", _F),
    ("thermal", _I), ("phase_change", _I), ("wall_thermal_bc", _I), ("heater_power", _F),
    ("conductivity_scale", _F), ("lee_evaporation", _F), ("lee_condensation", _F), ("thermo_mode", _I),
    ("vent_relaxation", _F), ("merge_ratio", _F), ("split_ratio", _F), ("max_transfer_fraction", _F),
    ("phase_change_density_limit", _F), ("vapor_mass_rebalance", _F),
    ("cfl", _F), ("viscous_number", _F), ("force_number", _F), ("capillary_number", _F),
    ("thermal_number", _F), ("dt_max", _F), ("dt_min", _F), ("fixed_dt", _F),
]


class Config(C.Structure):
    _fields_ = CONFIG_FIELDS

    def update(self, **kw):
        for k, v in kw.items():
            if k == "gravity":
                self.gravity[:] = [float(a) for a in v]
            else:
                if not hasattr(self, k):
                    raise AttributeError(k)
                setattr(self, k, int(v) if isinstance(v, bool) else v)
        return self


_D = C.c_double
DIAG_FIELDS = [
    ("time", _D), ("step", C.c_longlong), ("dt", _D),
    ("n_total", _I), ("n_liquid", _I), ("n_vapor", _I), ("n_wall", _I),
    ("mass_liquid", _D), ("mass_vapor", _D), ("mass_total", _D),
    ("kinetic_energy", _D), ("enthalpy", _D), ("heat_input", _D),
    ("evaporated_mass", _D), ("condensed_mass", _D), ("vented_mass", _D), ("vented_enthalpy", _D),
    ("T_sat", _D), ("p_ullage", _D), ("max_speed", _D),
    ("T_liquid_mean", _D), ("T_liquid_max", _D), ("T_vapor_mean", _D),
    ("liquid_com", _F * 3), ("liquid_momentum", _F * 3),
    ("splits", _I), ("merges", _I),
    ("slosh_force", _F * 3), ("slosh_moment", _F * 3),
    ("frame_acceleration", _F * 3), ("frame_angular_velocity", _F * 3),
]


class Diagnostics(C.Structure):
    _fields_ = DIAG_FIELDS

    def as_dict(self):
        out = {}
        for name, typ in DIAG_FIELDS:
            v = getattr(self, name)
            out[name] = tuple(float(a) for a in v) if isinstance(v, C.Array) else v
        return out


class HostParticles(C.Structure):
    _fields_ = [("n", _I), ("x", C.c_void_p), ("v", C.c_void_p), ("nrm", C.c_void_p), ("m", C.c_void_p),
                ("rho", C.c_void_p), ("T", C.c_void_p), ("phase", C.c_void_p), ("flags", C.c_void_p),
                ("id", C.c_void_p)]


class HostParticlesOut(C.Structure):
    _fields_ = [("n", C.c_int), ("x", C.c_void_p), ("v", C.c_void_p), ("nrm", C.c_void_p), ("m", C.c_void_p),
                ("rho", C.c_void_p), ("T", C.c_void_p), ("phase", C.c_void_p), ("flags", C.c_void_p),
                ("id", C.c_void_p)]


class CryoError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def host_particles(arrays: dict, keep: list):
    """Packs a dict of numpy arrays into a HostParticles struct.  `keep`
    receives the converted arrays so they outlive the call."""
    def conv(name, dtype, shape_last=None):
        a = arrays.get(name)
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dtype)
        keep.append(a)
        return a
    x = conv("x", np.float32)
    hp = HostParticles()
    hp.n = int(x.shape[0])
    hp.x = _ptr(x)
    hp.v = _ptr(conv("v", np.float32))
    hp.nrm = _ptr(conv("nrm", np.float32))
    hp.m = _ptr(conv("m", np.float32))
    hp.rho = _ptr(conv("rho", np.float32))
    hp.T = _ptr(conv("T", np.float32))
    hp.phase = _ptr(conv("phase", np.uint8))
    hp.flags = _ptr(conv("flags", np.uint8))
    hp.id = _ptr(conv("id", np.uint32))
    return hp


def field_dtype(name, real=np.float32):
    if name in U8_FIELDS:
        return np.uint8
    if name in U32_FIELDS:
        return np.uint32
    return real


def field_shape(name, n):
    return (n, 3) if name in VEC_FIELDS else (n,)


# SolverConfig defaults (sph_solver.hpp:20-91); cryo_config_default() in the
# library returns the same values (checked by the CPU tests).
CONFIG_DEFAULTS = dict(
    dx=0.005, h_factor=1.3, kernel=1, density_mode=0, normalize_initial_masses=1, gravity=(0.0, 0.0, -9.81),
    velocity_scale=0.0, sound_speed=0.0, tait_gamma=7.0, background_pressure=-1.0, vapor_stiffness=-1.0,
    clamp_negative_pressure=0, transport_velocity=1, transport_background_factor=2.0, transport_stress=0,
    transport_interface_only=1, particle_shifting=0, shifting_strength=0.25, artificial_viscosity=0.02,
    artificial_viscosity_vapor=0.2, delta_sph=0.1, no_slip=1, sps_turbulence=0, smagorinsky_cs=0.12,
    surface_tension=1, contact_angle_deg=90.0, contact_angle_wall_weight=0.01, wall_colour=1, wetting_model=0,
    csf_smooth_normals=0, csf_balanced=0, akinci_gamma=-1.0, akinci_beta=-1.0, thermal=1, phase_change=1,
    wall_thermal_bc=0, heater_power=0.0, conductivity_scale=1.0, lee_evaporation=10.0, lee_condensation=10.0,
    thermo_mode=0, vent_relaxation=0.02, merge_ratio=0.3, split_ratio=2.0, max_transfer_fraction=0.25,
    phase_change_density_limit=0.01, vapor_mass_rebalance=1.0, cfl=0.25, viscous_number=0.125,
    force_number=0.25, capillary_number=0.25, thermal_number=0.1, dt_max=1e-2, dt_min=1e-9, fixed_dt=0.0)

# Fluid presets (fluid_properties.cpp:16-79).
FLUID_PRESETS = {
    FLUID_LH2: dict(rho_liquid=70.85, rho_vapor=1.338, mu_liquid=1.33e-5, mu_vapor=1.11e-6, k_liquid=0.1034,
                    k_vapor=0.0166, cp_liquid=9770.0, cp_vapor=12200.0, sigma=1.93e-3, h_fg=445.6e3, T_sat=20.37,
                    p_sat=101325.0, R_gas=4124.2),
    FLUID_LN2: dict(rho_liquid=806.1, rho_vapor=4.61, mu_liquid=1.61e-4, mu_vapor=5.4e-6, k_liquid=0.1446,
                    k_vapor=0.0074, cp_liquid=2042.0, cp_vapor=1123.0, sigma=8.85e-3, h_fg=199.2e3, T_sat=77.36,
                    p_sat=101325.0, R_gas=296.8),
    FLUID_LOX: dict(rho_liquid=1141.0, rho_vapor=4.47, mu_liquid=1.96e-4, mu_vapor=6.9e-6, k_liquid=0.152,
                    k_vapor=0.0084, cp_liquid=1699.0, cp_vapor=972.0, sigma=13.2e-3, h_fg=213.1e3, T_sat=90.19,
                    p_sat=101325.0, R_gas=259.8),
    FLUID_LCH4: dict(rho_liquid=422.4, rho_vapor=1.816, mu_liquid=1.17e-4, mu_vapor=4.4e-6, k_liquid=0.184,
                     k_vapor=0.0119, cp_liquid=3481.0, cp_vapor=2218.0, sigma=13.4e-3, h_fg=510.8e3, T_sat=111.67,
                     p_sat=101325.0, R_gas=518.3),
    FLUID_H2O: dict(rho_liquid=998.2, rho_vapor=0.598, mu_liquid=1.0e-3, mu_vapor=1.23e-5, k_liquid=0.598,
                    k_vapor=0.0248, cp_liquid=4182.0, cp_vapor=2080.0, sigma=0.0728, h_fg=2.257e6, T_sat=373.15,
                    p_sat=101325.0, R_gas=461.5),
    FLUID_CUSTOM: dict(rho_liquid=1000.0, rho_vapor=1.0, mu_liquid=1e-3, mu_vapor=1e-5, k_liquid=0.6,
                       k_vapor=0.025, cp_liquid=4180.0, cp_vapor=2000.0, sigma=0.072, h_fg=2.26e6, T_sat=373.15,
                       p_sat=101325.0, R_gas=461.5),
}


def py_config(**kw):
    """Config filled from CONFIG_DEFAULTS (no library needed)."""
    c = Config()
    c.update(**CONFIG_DEFAULTS)
    return c.update(**kw)


def py_fluid(which):
    f = Fluid()
    for k, v in FLUID_PRESETS[which].items():
        setattr(f, k, v)
    return f


_lib = None


def lib_path():
    return os.path.join(HERE, LIB_NAME)


def load(path=None):
    """Loads libcryosph_b200.so and declares the entry points (idempotent)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or lib_path()
    if not os.path.exists(p):
        raise ImportError(f"{LIB_NAME} is not built (expected at {p}); run build.py")
    L = C.CDLL(p)
    vp, ip, i, f, d = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_float, C.c_double
    fp, dp = C.POINTER(C.c_float), C.POINTER(C.c_double)
    decl = {
        "cryo_abi_version": (i, []),
        "cryo_config_default": (None, [C.POINTER(Config)]),
        "cryo_fluid_preset": (i, [i, C.POINTER(Fluid)]),
        "cryo_saturation_temperature": (f, [C.POINTER(Fluid), f]),
        "cryo_saturation_pressure": (f, [C.POINTER(Fluid), f]),
        "cryo_create": (i, [C.POINTER(Config), C.POINTER(Fluid), i, C.POINTER(vp)]),
        "cryo_destroy": (None, [vp]),
        "cryo_last_error": (C.c_char_p, [vp]),
        "cryo_device_name": (i, [i, C.c_char_p, i]),
        "cryo_device_count": (i, []),
        "cryo_stream": (C.c_size_t, [vp]),
        "cryo_set_particles": (i, [vp, C.POINTER(HostParticles), fp, fp]),
        "cryo_step": (i, [vp]),
        "cryo_run_steps": (i, [vp, C.c_longlong]),
        "cryo_run_until": (i, [vp, d]),
        "cryo_relax": (i, [vp, d, f]),
        "cryo_next_dt": (i, [vp, dp]),
        "cryo_synchronize": (i, [vp]),
        "cryo_time": (i, [vp, dp, C.POINTER(C.c_longlong), dp]),
        "cryo_num_particles": (i, [vp, ip]),
        "cryo_capacity": (i, [vp, ip]),
        "cryo_diagnostics": (i, [vp, C.POINTER(Diagnostics)]),
        "cryo_diagnostics_request": (i, [vp]),
        "cryo_diagnostics_fetch": (i, [vp, C.POINTER(Diagnostics), i, ip]),
        "cryo_download": (i, [vp, vp]),
        "cryo_get_field": (i, [vp, i, vp, C.c_size_t]),
        "cryo_set_field": (i, [vp, i, vp, C.c_size_t]),
        "cryo_set_gravity": (i, [vp, fp]),
        "cryo_set_frame_motion": (i, [vp, fp, fp, fp, fp]),
        "cryo_set_maneuver": (i, [vp, i, dp, fp, fp, fp]),
        "cryo_clear_frame_motion": (i, [vp]),
        "cryo_set_heater_power": (i, [vp, f]),
        "cryo_set_contact_angle": (i, [vp, f]),
        "cryo_damp_velocities": (i, [vp, f]),
        "cryo_maneuver_evaluate": (i, [i, dp, fp, fp, d, fp, fp, fp]),
        "cryo_probe_pressure": (i, [vp, fp, i, fp]),
        "cryo_probe_pressure_noalloc": (i, [vp, fp, i, fp]),
        "cryo_sound_speed": (i, [vp, fp]),
        "cryo_smoothing_length": (i, [vp, fp]),
        "cryo_pass": (i, [vp, i]),
        "cryo_grid_info": (i, [vp, ip, ip, ip, ip, fp, fp]),
        "cryo_grid_tables": (i, [vp, vp, vp, vp, vp]),
        "cryo_neighbor_lists": (i, [vp, vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "cryo_stored_neighbor_lists": (i, [vp, vp, vp, C.c_longlong, C.POINTER(C.c_longlong)]),
        "cryo_set_pass_dt": (i, [vp, f]),
        "cryo_device_status": (i, [vp, C.POINTER(C.c_uint)]),
        "cryo_state_size": (i, [vp, C.POINTER(C.c_size_t)]),
        "cryo_save_state": (i, [vp, vp, C.c_size_t]),
        "cryo_load_state": (i, [vp, vp, C.c_size_t]),
        "cryo_set_graph_mode": (i, [vp, i]),
        "cryo_set_neighbor_mode": (i, [vp, i]),
        "cryo_set_field_arithmetic": (i, [vp, i]),
        "cryo_jitter_fluid": (i, [vp, f, C.c_ulonglong]),
        "cryo_field_arithmetic": (i, [vp, ip]),
        "cryo_adj_forward": (i, [vp, C.c_longlong, i, vp]),
        "cryo_adj_backward": (i, [vp, vp, vp, vp]),
        "cryo_adj_seed_state": (i, [vp, i, vp, C.c_size_t]),
        "cryo_adj_state_gradient": (i, [vp, i, vp, C.c_size_t]),
        "cryo_adj_memory": (i, [vp, C.POINTER(C.c_size_t)]),
        "cryo_adj_release": (i, [vp]),
        "cryo_set_surface_tension": (i, [vp, f]),
        "cryo_set_lee_coefficients": (i, [vp, f, f]),
        "cryo_slab_partition": (i, [C.POINTER(C.c_longlong), i, i, i, ip]),
        "cryo_slabs_create": (i, [C.POINTER(Config), C.POINTER(Fluid), i, ip, C.POINTER(vp)]),
        "cryo_slabs_destroy": (None, [vp]),
        "cryo_slabs_last_error": (C.c_char_p, [vp]),
        "cryo_slabs_count": (i, [vp, ip]),
        "cryo_slabs_set_particles": (i, [vp, C.POINTER(HostParticles), fp, fp]),
        "cryo_slabs_run_steps": (i, [vp, C.c_longlong]),
        "cryo_slabs_set_graph_mode": (i, [vp, i]),
        "cryo_slabs_graph_mode": (i, [vp, ip]),
        "cryo_slabs_num_particles": (i, [vp, ip]),
        "cryo_slabs_download": (i, [vp, C.POINTER(HostParticlesOut)]),
        "cryo_slabs_diagnostics": (i, [vp, C.POINTER(Diagnostics)]),
        "cryo_slabs_layout": (i, [vp, ip, ip, ip]),
    }
    for name, (res, args) in decl.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def config_default(lib=None, **kw):
    L = lib or load()
    c = Config()
    L.cryo_config_default(C.byref(c))
    return c.update(**kw)


def fluid_preset(which, lib=None):
    L = lib or load()
    f = Fluid()
    rc = L.cryo_fluid_preset(which, C.byref(f))
    if rc:
        raise CryoError(rc, "unknown fluid preset")
    return f


def vec3(v):
    return (C.c_float * 3)(*[float(a) for a in v])


def jitter_offsets(ids, seed, amplitude):
    """The offsets cryo_jitter_fluid adds on the device, restated on the host:
    (n, 3) float32, amplitude * (2u - 1) with u = the top 24 bits of the
    SplitMix64 output function of seed + (3 id + axis + 1) * 0x9E3779B97F4A7C15,
    scaled by 2^-24.  Apply them to liquid and vapour particles only."""
    ids = np.asarray(ids, np.uint64)
    with np.errstate(over="ignore"):
        k = (np.uint64(3) * ids)[:, None] + np.arange(1, 4, dtype=np.uint64)[None, :]
        z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u = (z >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)
    return np.float32(amplitude) * (np.float32(2.0) * u - np.float32(1.0))


class Context:
    """Thin RAII wrapper over a cryo_ctx (used by the parity tests)."""

    def __init__(self, cfg: Config, fluid: Fluid, device=0, lib=None):
        self.L = lib or load()
        self.h = C.c_void_p()
        rc = self.L.cryo_create(C.byref(cfg), C.byref(fluid), device, C.byref(self.h))
        if rc:
            raise CryoError(rc, "cryo_create failed")

    def close(self):
        if self.h:
            self.L.cryo_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != CRYO_OK:
            msg = self.L.cryo_last_error(self.h)
            raise CryoError(rc, msg.decode() if msg else "")

    def set_particles(self, arrays, lo, hi):
        keep = []
        hp = host_particles(arrays, keep)
        self.check(self.L.cryo_set_particles(self.h, C.byref(hp), vec3(lo), vec3(hi)))

    def num_particles(self):
        n = C.c_int()
        self.check(self.L.cryo_num_particles(self.h, C.byref(n)))
        return n.value

    def field(self, name):
        n = self.num_particles()
        out = np.empty(field_shape(name, n), dtype=field_dtype(name))
        self.check(self.L.cryo_get_field(self.h, FIELD_ID[name], out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def set_field(self, name, data):
        n = self.num_particles()
        a = np.ascontiguousarray(data, dtype=field_dtype(name)).reshape(field_shape(name, n))
        self.check(self.L.cryo_set_field(self.h, FIELD_ID[name], a.ctypes.data_as(C.c_void_p), a.nbytes))

    def set_neighbor_mode(self, use_lists):
        self.check(self.L.cryo_set_neighbor_mode(self.h, int(bool(use_lists))))

    def jitter_fluid(self, amplitude, seed):
        self.check(self.L.cryo_jitter_fluid(self.h, float(amplitude), int(seed)))

    def set_field_arithmetic(self, mode):
        """CRYO_ARITH_EXACT (0, the reference's IEEE sequence) or CRYO_ARITH_FAST (1)."""
        self.check(self.L.cryo_set_field_arithmetic(self.h, int(mode)))

    def device_status(self):
        st = C.c_uint()
        self.check(self.L.cryo_device_status(self.h, C.byref(st)))
        return st.value

    def set_graph_mode(self, on):
        self.check(self.L.cryo_set_graph_mode(self.h, int(bool(on))))

    def run_until(self, t):
        self.check(self.L.cryo_run_until(self.h, float(t)))

    def run_pass(self, name):
        self.check(self.L.cryo_pass(self.h, PASS_ID[name]))

    def set_pass_dt(self, dt):
        self.check(self.L.cryo_set_pass_dt(self.h, float(dt)))

    def step(self, n=1):
        self.check(self.L.cryo_run_steps(self.h, int(n)))

    def relax(self, duration, damping=0.98):
        self.check(self.L.cryo_relax(self.h, float(duration), float(damping)))

    def next_dt(self):
        d = C.c_double()
        self.check(self.L.cryo_next_dt(self.h, C.byref(d)))
        return d.value

    def diagnostics(self):
        d = Diagnostics()
        self.check(self.L.cryo_diagnostics(self.h, C.byref(d)))
        return d

    def request_diagnostics(self):
        self.check(self.L.cryo_diagnostics_request(self.h))

    def fetch_diagnostics(self, wait=True):
        """The oldest requested Diagnostics, or None (not ready / none pending)."""
        d, got = Diagnostics(), C.c_int()
        self.check(self.L.cryo_diagnostics_fetch(self.h, C.byref(d), 1 if wait else 0, C.byref(got)))
        return d if got.value else None

    def time(self):
        t, s, dt = C.c_double(), C.c_longlong(), C.c_double()
        self.check(self.L.cryo_time(self.h, C.byref(t), C.byref(s), C.byref(dt)))
        return t.value, s.value, dt.value

    def grid_info(self):
        nc, nx, ny, nz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        o, cell = (C.c_float * 3)(), C.c_float()
        self.check(self.L.cryo_grid_info(self.h, C.byref(nc), C.byref(nx), C.byref(ny), C.byref(nz), o,
                                         C.byref(cell)))
        return dict(num_cells=nc.value, nx=nx.value, ny=ny.value, nz=nz.value, origin=tuple(o), cell=cell.value)

    def grid_tables(self):
        info = self.grid_info()
        n = self.num_particles()
        keys = np.empty(n, np.uint32)
        perm = np.empty(n, np.uint32)
        cs = np.empty(info["num_cells"], np.int32)
        ce = np.empty(info["num_cells"], np.int32)
        self.check(self.L.cryo_grid_tables(self.h, _ptr(keys), _ptr(perm), _ptr(cs), _ptr(ce)))
        return keys, perm, cs, ce

    def neighbor_lists(self, stored=False):
        """(counts, concatenated lists) in reference order.  stored=True reads
        the stored lists the passes walk (walls: fluid neighbours only)."""
        fn = self.L.cryo_stored_neighbor_lists if stored else self.L.cryo_neighbor_lists
        n = self.num_particles()
        counts = np.empty(n, np.int32)
        total = C.c_longlong()
        self.check(fn(self.h, _ptr(counts), None, 0, C.byref(total)))
        lst = np.empty(max(total.value, 1), np.int32)
        self.check(fn(self.h, _ptr(counts), _ptr(lst), total.value, C.byref(total)))
        return counts, lst[: total.value]

    def probe_pressure(self, pts):
        """Solver::probe_pressure: Shepard liquid pressure at each point (NaN where dry)."""
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        out = np.empty(len(pts), np.float32)
        self.check(self.L.cryo_probe_pressure(self.h, pts.ctypes.data_as(C.POINTER(C.c_float)), len(pts),
                                              out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_frame_motion(self, a=(0, 0, 0), w=(0, 0, 0), wd=(0, 0, 0), o=(0, 0, 0)):
        self.check(self.L.cryo_set_frame_motion(self.h, vec3(a), vec3(w), vec3(wd), vec3(o)))

    # ---------------------------------------------- differentiated window
    ADJ_STATE = {"x": 0, "v": 1, "T": 2, "m": 3, "a": 4, "ab": 5}

    def set_surface_tension(self, sigma):
        self.check(self.L.cryo_set_surface_tension(self.h, float(sigma)))

    def set_lee_coefficients(self, evaporation, condensation):
        self.check(self.L.cryo_set_lee_coefficients(self.h, float(evaporation), float(condensation)))

    def set_contact_angle(self, degrees):
        self.check(self.L.cryo_set_contact_angle(self.h, float(degrees)))

    def set_heater_power(self, watts):
        self.check(self.L.cryo_set_heater_power(self.h, float(watts)))

    def adj_forward(self, steps, checkpoint_every=20):
        """Runs the window; returns [int F (3), int M (3), p_ullage]."""
        out = np.zeros(7, np.float64)
        self.check(self.L.cryo_adj_forward(self.h, int(steps), int(checkpoint_every), _ptr(out)))
        self._adj_steps = int(steps)
        return out

    def adj_seed_state(self, name, data):
        comps = 1 if name in ("T", "m") else 3
        a = np.ascontiguousarray(data, np.float32).reshape(-1)
        self.check(self.L.cryo_adj_seed_state(self.h, self.ADJ_STATE[name], _ptr(a), a.size))

    def adj_backward(self, seed):
        """Returns (grads[5]: sigma, contact angle (deg), lee_evap, lee_cond,
        heater power; frame acceleration gradient per step (steps, 3))."""
        sd = np.ascontiguousarray(seed, np.float64).reshape(7)
        g = np.zeros(5, np.float64)
        fg = np.zeros((self._adj_steps, 3), np.float64)
        self.check(self.L.cryo_adj_backward(self.h, _ptr(sd), _ptr(g), _ptr(fg)))
        return g, fg

    def adj_state_gradient(self, name):
        comps = 1 if name in ("T", "m") else 3
        n = self.num_particles()
        out = np.empty(n * comps, np.float32)
        self.check(self.L.cryo_adj_state_gradient(self.h, self.ADJ_STATE[name], _ptr(out), out.size))
        return out if comps == 1 else out.reshape(n, 3)

    def adj_memory(self):
        b = C.c_size_t()
        self.check(self.L.cryo_adj_memory(self.h, C.byref(b)))
        return b.value


def slab_partition(layer_counts, nslabs, min_layers=3, lib=None):
    """Layer boundaries of cryo_slab_partition (host arithmetic only)."""
    L = lib or load()
    counts = np.ascontiguousarray(layer_counts, dtype=np.int64)
    out = np.zeros(nslabs + 1, dtype=np.int32)
    rc = L.cryo_slab_partition(counts.ctypes.data_as(C.POINTER(C.c_longlong)), int(counts.size), int(nslabs),
                               int(min_layers), out.ctypes.data_as(C.POINTER(C.c_int)))
    if rc != CRYO_OK:
        raise CryoError(rc, "cryo_slab_partition: bad arguments")
    return out


class Slabs:
    """One tank cut into slabs of cell layers (cryo_slabs_*), each slab a
    context on devices[r]."""

    def __init__(self, cfg: Config, fluid: Fluid, nslabs, devices=None, lib=None):
        self.L = lib or load()
        self.h = C.c_void_p()
        devs = None
        if devices is not None:
            self._devs = (C.c_int * nslabs)(*[int(d) for d in devices])
            devs = self._devs
        rc = self.L.cryo_slabs_create(C.byref(cfg), C.byref(fluid), int(nslabs), devs, C.byref(self.h))
        if rc:
            msg = self.L.cryo_slabs_last_error(None)
            raise CryoError(rc, msg.decode() if msg else "cryo_slabs_create failed")
        self.nslabs = int(nslabs)

    def close(self):
        if self.h:
            self.L.cryo_slabs_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != CRYO_OK:
            msg = self.L.cryo_slabs_last_error(self.h)
            raise CryoError(rc, msg.decode() if msg else "")

    def set_particles(self, arrays, lo, hi):
        keep = []
        hp = host_particles(arrays, keep)
        self.check(self.L.cryo_slabs_set_particles(self.h, C.byref(hp), vec3(lo), vec3(hi)))

    def step(self, n=1):
        self.check(self.L.cryo_slabs_run_steps(self.h, int(n)))

    def set_graph_mode(self, on):
        self.check(self.L.cryo_slabs_set_graph_mode(self.h, 1 if on else 0))

    def graph_mode(self):
        """0 off, 1 the steps replay the group graph, 2 on but the capture was refused."""
        m = C.c_int()
        self.check(self.L.cryo_slabs_graph_mode(self.h, C.byref(m)))
        return m.value

    def num_particles(self):
        n = C.c_int()
        self.check(self.L.cryo_slabs_num_particles(self.h, C.byref(n)))
        return n.value

    def particles(self):
        n = self.num_particles()
        out = {"x": np.empty((n, 3), np.float32), "v": np.empty((n, 3), np.float32),
               "nrm": np.empty((n, 3), np.float32), "m": np.empty(n, np.float32), "rho": np.empty(n, np.float32),
               "T": np.empty(n, np.float32), "phase": np.empty(n, np.uint8), "flags": np.empty(n, np.uint8),
               "id": np.empty(n, np.uint32)}
        o = HostParticlesOut(n, *[_ptr(out[k]) for k in ("x", "v", "nrm", "m", "rho", "T", "phase", "flags", "id")])
        self.check(self.L.cryo_slabs_download(self.h, C.byref(o)))
        return out

    def diagnostics(self):
        d = Diagnostics()
        self.check(self.L.cryo_slabs_diagnostics(self.h, C.byref(d)))
        return d

    def layout(self):
        zb = np.zeros(self.nslabs + 1, np.int32)
        owned = np.zeros(self.nslabs, np.int32)
        held = np.zeros(self.nslabs, np.int32)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self.check(self.L.cryo_slabs_layout(self.h, ip(zb), ip(owned), ip(held)))
        return zb, owned, held
