"""Struct layouts and constants of include/cryosph_b200.h for the checkers
(TEST INFRASTRUCTURE ONLY).

The reference driver (ref_driver.h) and the oracle (cryo_oracle.h) take the
same POD structs as the product's C ABI: cryo_config_t, cryo_fluid_t,
cryo_diagnostics_t, cryo_host_particles_t.  This module declares them for
ctypes on its own, so that the checkers -- and bench.py's reference arm in
particular -- load nothing from the package: a process that times the
reference maps only oracle/_ref.  tests/test_oracle.py checks that every
layout here equals the package's (cryo_cabi) field for field.

The SolverConfig defaults follow sph_solver.hpp:20-91 of the reference and
the fluid presets fluid_properties.cpp:16-79.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

LIQUID, VAPOR, WALL, DEAD = 0, 1, 2, 3
FLUID_CUSTOM, FLUID_LH2, FLUID_LN2, FLUID_LOX, FLUID_LCH4, FLUID_H2O = range(6)

# CRYO_F_* field ids and CRYO_PASS_* pass ids, in header order
FIELDS = [
    "x", "v", "vt", "nrm", "m", "m0", "rho", "T", "phase", "flags", "id",
    "a", "ab", "fw", "mw", "ns", "vw",
    "p", "drho", "dTdt", "sigma", "kappa", "nu_t", "alpha",
    "wall_w", "heat_w", "out_m", "out_h", "w_norm", "rmin", "p_wv",
]
FIELD_ID = {name: k for k, name in enumerate(FIELDS)}
VEC_FIELDS = {"x", "v", "vt", "nrm", "a", "ab", "fw", "mw", "ns", "vw"}
PASSES = [
    "kick_drift", "grid_build", "density", "normalize_masses", "eos", "wall_boundary", "interface",
    "transport", "sps", "momentum", "smooth_normals", "csf", "akinci", "density_rate", "thermal",
    "maxima", "kick", "shifting", "pc_sources", "pc_normalize", "pc_apply", "rebalance", "split",
    "venting", "saturation",
]
PASS_ID = {name: k for k, name in enumerate(PASSES)}

_F, _I, _D = C.c_float, C.c_int, C.c_double


class Fluid(C.Structure):
    _fields_ = [(n, _F) for n in ("rho_liquid", "rho_vapor", "mu_liquid", "mu_vapor", "k_liquid", "k_vapor",
                                  "cp_liquid", "cp_vapor", "sigma", "h_fg", "T_sat", "p_sat", "R_gas")]


# cryo_config_t: (name, ctype, default)
_CONFIG = [
    ("dx", _F, 0.005), ("h_factor", _F, 1.3), ("kernel", _I, 1), ("density_mode", _I, 0),
    ("normalize_initial_masses", _I, 1), ("gravity", _F * 3, (0.0, 0.0, -9.81)), ("velocity_scale", _F, 0.0),
    ("sound_speed", _F, 0.0), ("tait_gamma", _F, 7.0), ("background_pressure", _F, -1.0),
    ("vapor_stiffness", _F, -1.0), ("clamp_negative_pressure", _I, 0), ("transport_velocity", _I, 1),
    ("transport_background_factor", _F, 2.0), ("transport_stress", _I, 0), ("transport_interface_only", _I, 1),
    ("particle_shifting", _I, 0), ("shifting_strength", _F, 0.25), ("artificial_viscosity", _F, 0.02),
    ("artificial_viscosity_vapor", _F, 0.2), ("delta_sph", _F, 0.1), ("no_slip", _I, 1),
    ("sps_turbulence", _I, 0), ("smagorinsky_cs", _F, 0.12), ("surface_tension", _I, 1),
    ("contact_angle_deg", _F, 90.0), ("contact_angle_wall_weight", _F, 0.01), ("wall_colour", _I, 1),
    ("wetting_model", _I, 0), ("csf_smooth_normals", _I, 0), ("csf_balanced", _I, 0), ("akinci_gamma", _F, -1.0),
    ("akinci_beta", _F, -1.0), ("thermal", _I, 1), ("phase_change", _I, 1), ("wall_thermal_bc", _I, 0),
    ("heater_power", _F, 0.0), ("conductivity_scale", _F, 1.0), ("lee_evaporation", _F, 10.0),
    ("lee_condensation", _F, 10.0), ("thermo_mode", _I, 0), ("vent_relaxation", _F, 0.02),
    ("merge_ratio", _F, 0.3), ("split_ratio", _F, 2.0), ("max_transfer_fraction", _F, 0.25),
    ("phase_change_density_limit", _F, 0.01), ("vapor_mass_rebalance", _F, 1.0), ("cfl", _F, 0.25),
    ("viscous_number", _F, 0.125), ("force_number", _F, 0.25), ("capillary_number", _F, 0.25),
    ("thermal_number", _F, 0.1), ("dt_max", _F, 1e-2), ("dt_min", _F, 1e-9), ("fixed_dt", _F, 0.0),
]
CONFIG_DEFAULTS = {name: default for name, _, default in _CONFIG}


class Config(C.Structure):
    _fields_ = [(name, typ) for name, typ, _ in _CONFIG]

    def update(self, **kw):
        for k, v in kw.items():
            if k == "gravity":
                self.gravity[:] = [float(a) for a in v]
            elif not hasattr(self, k):
                raise AttributeError(k)
            else:
                setattr(self, k, int(v) if isinstance(v, bool) else v)
        return self


class Diagnostics(C.Structure):
    _fields_ = [
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

    def as_dict(self):
        return {name: (tuple(float(a) for a in getattr(self, name)) if isinstance(getattr(self, name), C.Array)
                       else getattr(self, name)) for name, _ in self._fields_}


class HostParticles(C.Structure):
    _fields_ = [("n", _I)] + [(k, C.c_void_p) for k in ("x", "v", "nrm", "m", "rho", "T", "phase", "flags", "id")]


class HostOut(C.Structure):
    """cryo_host_particles_out_t as the reference driver fills it."""
    _fields_ = [("n", _I), ("x", C.POINTER(_F)), ("v", C.POINTER(_F)), ("nrm", C.POINTER(_F)),
                ("m", C.POINTER(_F)), ("rho", C.POINTER(_F)), ("T", C.POINTER(_F)),
                ("phase", C.POINTER(C.c_uint8)), ("flags", C.POINTER(C.c_uint8)), ("id", C.POINTER(C.c_uint32))]


class RefError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


FLUID_PRESETS = {
    FLUID_LH2: (70.85, 1.338, 1.33e-5, 1.11e-6, 0.1034, 0.0166, 9770.0, 12200.0, 1.93e-3, 445.6e3, 20.37,
                101325.0, 4124.2),
    FLUID_LN2: (806.1, 4.61, 1.61e-4, 5.4e-6, 0.1446, 0.0074, 2042.0, 1123.0, 8.85e-3, 199.2e3, 77.36, 101325.0,
                296.8),
    FLUID_LOX: (1141.0, 4.47, 1.96e-4, 6.9e-6, 0.152, 0.0084, 1699.0, 972.0, 13.2e-3, 213.1e3, 90.19, 101325.0,
                259.8),
    FLUID_LCH4: (422.4, 1.816, 1.17e-4, 4.4e-6, 0.184, 0.0119, 3481.0, 2218.0, 13.4e-3, 510.8e3, 111.67, 101325.0,
                 518.3),
    FLUID_H2O: (998.2, 0.598, 1.0e-3, 1.23e-5, 0.598, 0.0248, 4182.0, 2080.0, 0.0728, 2.257e6, 373.15, 101325.0,
                461.5),
    FLUID_CUSTOM: (1000.0, 1.0, 1e-3, 1e-5, 0.6, 0.025, 4180.0, 2000.0, 0.072, 2.26e6, 373.15, 101325.0, 461.5),
}


def config(**kw):
    """cryo_config_t with the reference's SolverConfig defaults, then `kw`."""
    return Config().update(**CONFIG_DEFAULTS).update(**kw)


def fluid(which, **kw):
    f = Fluid()
    for (name, _), v in zip(Fluid._fields_, FLUID_PRESETS[which]):
        setattr(f, name, v)
    for k, v in kw.items():
        setattr(f, k, v)
    return f


def as_struct(cls, obj):
    """`obj` as an instance of `cls`: a struct of another module with the same
    layout (the package's cryo_cabi classes) is copied byte for byte."""
    if isinstance(obj, cls):
        return obj
    if C.sizeof(obj) != C.sizeof(cls):
        raise TypeError(f"{type(obj).__name__} does not have the layout of {cls.__name__}")
    return cls.from_buffer_copy(C.string_at(C.addressof(obj), C.sizeof(obj)))


def vec3(v):
    return (_F * 3)(*[float(a) for a in v])


def field_dtype(name, real=np.float32):
    if name in ("phase", "flags"):
        return np.uint8
    if name == "id":
        return np.uint32
    return real


def field_shape(name, n):
    return (n, 3) if name in VEC_FIELDS else (n,)


def host_particles(arrays, keep):
    """HostParticles over a dict of numpy arrays (x, v, nrm, m, rho, T, phase,
    flags, id); `keep` holds the converted arrays for the call's lifetime."""
    types = {"x": np.float32, "v": np.float32, "nrm": np.float32, "m": np.float32, "rho": np.float32,
             "T": np.float32, "phase": np.uint8, "flags": np.uint8, "id": np.uint32}
    hp = HostParticles()
    for name, dt in types.items():
        a = arrays.get(name)
        if a is None:
            continue
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        setattr(hp, name, a.ctypes.data_as(C.c_void_p))
    hp.n = int(np.asarray(arrays["x"]).shape[0])
    return hp
