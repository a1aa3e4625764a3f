"""Seeded synthetic inputs shared by the tests (and the golden-vector script).

Each scenario returns (config, fluid, particles, domain_lo, domain_hi): the
reference's own lattice generator (geometry.cpp:242-330, through the reference
build in oracle/_ref) fills the tank, fluid positions get a uniform
+-0.05 dx jitter from numpy PCG64(seed), walls stay on the lattice, and the
domain padding is Solver::build_tank's (sph_solver.cu:430-437).
"""
from __future__ import annotations

import numpy as np

import cryo_cabi as cabi
import refpy

SEED = 2002


def jitter(parts, dx, seed=SEED, amp=0.05):
    rng = np.random.Generator(np.random.PCG64(seed))
    fluid = parts["phase"] != cabi.WALL
    x = parts["x"].copy()
    x[fluid] += rng.uniform(-amp * dx, amp * dx, size=(int(fluid.sum()), 3)).astype(np.float32)
    out = dict(parts)
    out["x"] = x
    return out


def tank(nodes, fluid, dx, fill, seed=SEED, wall_layers=3):
    parts = refpy.tank_particles(nodes, fluid, dx, fill)
    lo, hi = refpy.tank_domain(nodes, dx, wall_layers)
    return jitter(parts, dx, seed), lo, hi


def c1(dx=0.004):
    """Closed LN2 cylinder R 0.05 H 0.12, fill 0.5, milli-g, 20 W heater."""
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=dx, gravity=(0, 0, -9.81e-4), heater_power=20.0, thermo_mode=1)
    parts, lo, hi = tank([(refpy.CYLINDER, 0, 0, (0.05, 0.12, 0))], fl, dx, refpy.make_fill(fill_fraction=0.5))
    return cfg, fl, parts, lo, hi


def box_split():
    """Closed LN2 box with superheat and a low split ratio (splits + evaporation)."""
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -0.5), contact_angle_deg=10, velocity_scale=1, thermo_mode=1,
                         lee_evaporation=5, lee_condensation=5, split_ratio=1.05)
    parts, lo, hi = tank([(refpy.BOX, 0, 0, (0.04, 0.04, 0.04))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.5, T_liquid=fl.T_sat + 3))
    return cfg, fl, parts, lo, hi


def vented():
    """Vented LN2 box (venting + condensation), contact-line force wetting."""
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, 0), contact_angle_deg=5, velocity_scale=1, thermo_mode=0,
                         vent_relaxation=0.2, lee_evaporation=2, lee_condensation=2, wetting_model=2,
                         wall_thermal_bc=1, heater_power=5.0)
    parts, lo, hi = tank([(refpy.BOX, 0, 0, (0.04, 0.04, 0.04))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.5, T_liquid=fl.T_sat + 3, T_vapor=fl.T_sat - 1))
    return cfg, fl, parts, lo, hi


def dam_break(dx=0.04):
    """Single-phase dam break with an obstacle (validation/spheric_test2/run.py:36-66),
    continuity density, free-slip walls, no surface tension or heat."""
    fl = cabi.py_fluid(cabi.FLUID_H2O)
    fl.mu_liquid = 1.0e-3
    cfg = cabi.py_config(dx=dx, gravity=(0, 0, -9.81), surface_tension=0, thermal=0, phase_change=0,
                         density_mode=1, velocity_scale=(2 * 9.81 * 0.55) ** 0.5, artificial_viscosity=0.02,
                         delta_sph=0.1, no_slip=0)
    x_front, box = 0.744, (0.161, 0.403, 0.161)
    nodes = [
        (refpy.BOX, 0, 0, (3.22, 1.0, 1.0)),
        (refpy.TRANSLATED, 0, 0, (1.61, 0.0, 0.5)),
        (refpy.BOX, 0, 0, box),
        (refpy.TRANSLATED, 2, 0, (x_front - box[0] / 2, 0.0, box[2] / 2)),
        (refpy.DIFFERENCE, 1, 3, (0, 0, 0)),
    ]
    fill = refpy.make_fill(mode=2)
    parts = refpy.tank_particles(nodes, fl, dx, fill)
    x, ph = parts["x"], parts["phase"]
    keep = (ph == 2) | ((x[:, 0] > 3.22 - 1.228) & (x[:, 2] < 0.55))
    parts = {k: v[keep] for k, v in parts.items()}
    parts["id"] = np.arange(len(parts["x"]), dtype=np.uint32)
    pad = 4 * dx
    lo, hi = (-pad, -0.5 - pad, -pad), (3.22 + pad, 0.5 + pad, 1.0 + pad)
    return cfg, fl, jitter(parts, dx), lo, hi


def akinci():
    """Liquid-only (free surface) water drop in a box with the Akinci model."""
    fl = cabi.py_fluid(cabi.FLUID_H2O)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -1.0), surface_tension=2, thermal=0, phase_change=0,
                         velocity_scale=0.5, contact_angle_deg=60)
    parts, lo, hi = tank([(refpy.BOX, 0, 0, (0.04, 0.04, 0.04))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.4, include_vapor=False))
    return cfg, fl, parts, lo, hi


def options():
    """Closed LN2 capsule exercising the optional paths: balanced CSF with
    smoothed normals, SPS, particle shifting, the cubic spline kernel,
    transport stress, both wetting models, isothermal walls."""
    fl = cabi.py_fluid(cabi.FLUID_LOX)
    cfg = cabi.py_config(dx=0.004, gravity=(0.02, 0, -0.1), kernel=0, csf_balanced=1, csf_smooth_normals=1,
                         sps_turbulence=1, particle_shifting=1, transport_stress=1, wetting_model=2,
                         wall_thermal_bc=1, thermo_mode=1, heater_power=2.0, velocity_scale=0.5,
                         contact_angle_deg=40)
    parts, lo, hi = tank([(refpy.CAPSULE, 0, 0, (0.02, 0.02, 0))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.6, T_liquid=fl.T_sat + 1))
    return cfg, fl, parts, lo, hi


def lh2_sphere():
    """The LH2 sphere physics on a small sphere: closed LH2 tank R 0.05 m, fill 0.5,
    1e-4 g (the LH2 sphere workload of R 0.5 m, scaled to a test size)."""
    fl = cabi.py_fluid(cabi.FLUID_LH2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1)
    parts, lo, hi = tank([(refpy.SPHERE, 0, 0, (0.05, 0, 0))], fl, 0.004, refpy.make_fill(fill_fraction=0.5))
    return cfg, fl, parts, lo, hi


def ln2_boiloff():
    """The LN2 boil-off physics on a small cylinder: closed LN2 tank R 0.03 m, H 0.075 m,
    fill 0.5, 2 K superheat, Lee coefficient 5, 20 W heater, 1e-4 g."""
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1, lee_evaporation=5, heater_power=20.0)
    parts, lo, hi = tank([(refpy.CYLINDER, 0, 0, (0.03, 0.075, 0))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.5, T_liquid=fl.T_sat + 2))
    return cfg, fl, parts, lo, hi


def lch4_box():
    """A closed methane tank with superheated liquid (one of the ensemble's fluid presets)."""
    fl = cabi.py_fluid(cabi.FLUID_LCH4)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1, lee_evaporation=2, lee_condensation=2,
                         velocity_scale=1, contact_angle_deg=20)
    parts, lo, hi = tank([(refpy.BOX, 0, 0, (0.04, 0.04, 0.04))], fl, 0.004,
                         refpy.make_fill(fill_fraction=0.3, T_liquid=fl.T_sat + 2))
    return cfg, fl, parts, lo, hi


SCENARIOS = {"c1": c1, "box_split": box_split, "vented": vented, "dam_break": dam_break, "akinci": akinci,
             "options": options, "lh2_sphere": lh2_sphere, "ln2_boiloff": ln2_boiloff, "lch4_box": lch4_box}


def normwise(a, b):
    """max |a - b| / max |b| (0 when both vanish)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    d = np.abs(a - b)
    fin = np.isfinite(b)
    if not np.array_equal(np.isfinite(a), fin):
        return np.inf
    scale = np.max(np.abs(b[fin])) if fin.any() else 0.0
    err = np.max(d[fin]) if fin.any() else 0.0
    if scale == 0.0:
        return float(err)
    return float(err / scale)


def assert_stored_lists(g, oc, ol, phase):
    """The stored neighbour lists the CUDA passes walk equal the oracle's
    lists (counts oc, concatenated lists ol), a wall's restricted to its
    fluid neighbours (phase <= 1)."""
    sc, sl = g.neighbor_lists(stored=True)
    parts = np.split(ol, np.cumsum(oc)[:-1]) if len(oc) else []
    want = [lst if phase[i] != 2 else lst[phase[lst] <= 1] for i, lst in enumerate(parts)]
    wc = np.array([len(w) for w in want], np.int32)
    assert np.array_equal(sc, wc), "stored neighbour list counts differ"
    if want:
        assert np.array_equal(sl, np.concatenate(want)), "stored neighbour lists differ (membership or order)"
