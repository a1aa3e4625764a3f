"""The CryoSPH Python module on the CPU side: the reference's public API
(tests/python/test_bindings.py of the reference, the parts that need no
device), and the lattice generator against the reference's own."""
import math

import numpy as np
import pytest

import CryoSPH as cs
import cryo_cabi as cabi
import refpy

needs_ref = pytest.mark.skipif(not refpy.ref_available(), reason="reference CPU build (oracle/_ref) not built")


def test_module_metadata():
    assert cs.__version__ == "0.2.0"
    assert isinstance(cs.cuda_backend, bool) and cs.cuda_backend
    assert isinstance(cs.device_name(), str) and cs.device_name()
    assert cs.double_precision is False


def test_fluid_presets_and_clausius_clapeyron():
    ln2 = cs.FluidProperties.liquid_nitrogen()
    assert ln2.name == "LN2"
    assert ln2.rho_liquid / ln2.rho_vapor > 100
    assert ln2.saturation_temperature(ln2.p_sat) == pytest.approx(ln2.T_sat, rel=1e-6)
    p2 = ln2.saturation_pressure(ln2.T_sat + 2.0)
    assert p2 > ln2.p_sat
    assert ln2.saturation_temperature(p2) == pytest.approx(ln2.T_sat + 2.0, rel=1e-5)
    for f in (cs.FluidProperties.liquid_hydrogen(), cs.FluidProperties.liquid_oxygen(),
              cs.FluidProperties.liquid_methane(), cs.FluidProperties.water()):
        assert f.rho_liquid > f.rho_vapor > 0
    assert "rho_l=" in repr(ln2)


def test_geometry_sdf():
    tank = cs.CylinderTank(radius=0.1, height=0.3)
    assert tank.sdf(0, 0, 0) == pytest.approx(-0.1)
    assert tank.volume() == pytest.approx(math.pi * 0.01 * 0.3)
    lo, hi = tank.bounds
    assert lo[2] == pytest.approx(-0.15) and hi[0] == pytest.approx(0.1)
    assert cs.SphereTank(0.5).sdf(0, 0, 0.5) == pytest.approx(0.0)
    assert cs.CapsuleTank(0.1, 0.2).volume() == pytest.approx(math.pi * 0.01 * 0.2 + 4 / 3 * math.pi * 1e-3)
    assert cs.BoxTank(1, 2, 3).volume() == pytest.approx(6.0)
    with pytest.raises(ValueError):
        cs.SphereTank(-1.0)


def test_csg_geometry():
    tank = cs.Translated(cs.BoxTank(0.1, 0.1, 0.1), (0.05, 0.0, 0.05))
    block = cs.Translated(cs.BoxTank(0.02, 0.02, 0.02), (0.05, 0.0, 0.01))
    geo = cs.Difference(tank, block)
    assert geo.sdf(0.05, 0.0, 0.01) > 0
    assert geo.sdf(0.02, 0.0, 0.05) < 0
    assert cs.Union(tank, block).sdf(0.05, 0.0, 0.01) < 0
    assert geo.name.startswith("difference(")


def test_mesh_tank_cube(tmp_path):
    verts = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    faces = [(1, 3, 2), (1, 4, 3), (5, 6, 7), (5, 7, 8), (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6),
             (3, 4, 8), (3, 8, 7), (4, 1, 5), (4, 5, 8)]
    p = tmp_path / "cube.obj"
    p.write_text("".join(f"v {a} {b} {c}\n" for a, b, c in verts) + "".join(f"f {a} {b} {c}\n" for a, b, c in faces))
    m = cs.MeshTank(str(p), scale=0.5)
    assert m.num_triangles == 12
    assert m.volume() == pytest.approx(1.0)
    assert m.sdf(0, 0, 0) == pytest.approx(-0.5)
    assert m.sdf(1.0, 0, 0) == pytest.approx(0.5)
    assert abs(m.winding_number(0, 0, 0)) == pytest.approx(1.0)
    assert m.winding_number(2, 2, 2) == pytest.approx(0.0, abs=1e-9)


def test_config_roundtrip():
    cfg = cs.SolverConfig()
    cfg.dx = 0.005
    cfg.gravity = (0.0, 0.0, 0.0)
    cfg.contact_angle_deg = 12.5
    cfg.surface_tension = cs.SurfaceTensionModel.Akinci
    assert cfg.gravity == (0.0, 0.0, 0.0)
    assert cfg.contact_angle_deg == 12.5
    assert cfg.surface_tension == cs.SurfaceTensionModel.Akinci
    d = cs.SolverConfig()
    assert d.h_factor == pytest.approx(1.3) and d.kernel == cs.KernelType.WendlandC2 and d.cfl == pytest.approx(0.25)


def test_bad_inputs_raise_before_the_device():
    ln2 = cs.FluidProperties.liquid_nitrogen()
    cfg = cs.SolverConfig()
    cfg.contact_angle_deg = 200.0
    with pytest.raises(ValueError):
        cs.Solver(cfg, ln2)
    cfg = cs.SolverConfig()
    cfg.dx = 0.0
    with pytest.raises(ValueError):
        cs.Solver(cfg, ln2)


def test_maneuver_profile():
    prof = cs.ManeuverProfile([0.0, 1.0], np.array([[0, 0, 0], [2.0, 0, 0]]),
                              np.array([[0, 0, 0], [0, 0, 1.0]]), origin=(0, 0, 0))
    a, w, wd = prof.evaluate(0.5)
    assert a == pytest.approx((1.0, 0.0, 0.0))
    assert w[2] == pytest.approx(0.5) and wd[2] == pytest.approx(1.0)
    with pytest.raises(ValueError):
        cs.ManeuverProfile([0.0, 0.0], np.zeros((2, 3)))
    with pytest.raises(ValueError):
        cs.ManeuverProfile([0.0, 1.0], np.zeros((3, 3)))


def test_make_block():
    p = cs.make_block((0, 0, 0), (0.02, 0.02, 0.01), 0.005, cs.Phase.Liquid, 1000.0, 300.0)
    assert p["position"].shape == (4 * 4 * 2, 3)
    assert np.allclose(p["mass"], 1000.0 * 0.005 ** 3)
    assert np.array_equal(p["id"], np.arange(32))


GEOMS = [
    ("cylinder", lambda: cs.CylinderTank(0.05, 0.12), [(refpy.CYLINDER, 0, 0, (0.05, 0.12, 0))], 0.004,
     dict(fill_fraction=0.5)),
    ("sphere", lambda: cs.SphereTank(0.1), [(refpy.SPHERE, 0, 0, (0.1, 0, 0))], 0.006, dict(fill_fraction=0.3)),
    ("capsule", lambda: cs.CapsuleTank(0.03, 0.04), [(refpy.CAPSULE, 0, 0, (0.03, 0.04, 0))], 0.004,
     dict(fill_fraction=0.7, heater_zmin=-0.01, heater_zmax=0.01)),
    ("bubble", lambda: cs.BoxTank(0.04, 0.05, 0.06), [(refpy.BOX, 0, 0, (0.04, 0.05, 0.06))], 0.004,
     dict(fill_fraction=0.5, mode=1, bubble=(0.005, 0, 0))),
    ("dam", lambda: cs.Difference(cs.Translated(cs.BoxTank(3.22, 1.0, 1.0), (1.61, 0.0, 0.5)),
                                  cs.Translated(cs.BoxTank(0.161, 0.403, 0.161), (0.744 - 0.0805, 0.0, 0.0805))),
     [(refpy.BOX, 0, 0, (3.22, 1.0, 1.0)), (refpy.TRANSLATED, 0, 0, (1.61, 0.0, 0.5)),
      (refpy.BOX, 0, 0, (0.161, 0.403, 0.161)), (refpy.TRANSLATED, 2, 0, (0.744 - 0.0805, 0.0, 0.0805)),
      (refpy.DIFFERENCE, 1, 3, (0, 0, 0))], 0.04, dict(mode=2)),
]


@needs_ref
@pytest.mark.parametrize("name,mk,nodes,dx,fillkw", GEOMS, ids=[g[0] for g in GEOMS])
def test_lattice_generator_bit_identical_to_reference(name, mk, nodes, dx, fillkw):
    ln2 = cs.FluidProperties.liquid_nitrogen()
    f = cs.FillSpec()
    rf_kw = {}
    for k, v in fillkw.items():
        if k == "mode":
            f.mode = [cs.FillMode.Settled, cs.FillMode.CentralBubble, cs.FillMode.Full][v]
            rf_kw["mode"] = v
        elif k == "bubble":
            f.bubble_center = v
            rf_kw["bubble"] = v
        else:
            setattr(f, k, v)
            rf_kw[k] = v
    ours = cs.tank_particles(mk(), ln2, dx, f)
    ref = refpy.tank_particles(nodes, cabi.py_fluid(cabi.FLUID_LN2), dx, refpy.make_fill(**rf_kw))
    keymap = {"position": "x", "velocity": "v", "normal": "nrm", "mass": "m", "density": "rho",
              "temperature": "T", "phase": "phase", "flags": "flags", "id": "id"}
    for k, v in keymap.items():
        a, b = np.asarray(ours[k]), np.asarray(ref[v])
        assert a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    lo, hi = cs.tank_domain(mk(), dx, 3)
    rlo, rhi = refpy.tank_domain(nodes, dx, 3)
    assert np.array_equal(np.float32(lo), np.float32(rlo)) and np.array_equal(np.float32(hi), np.float32(rhi))
