"""The CryoSPH Python module on the CPU side: the reference's public API
(tests/python/test_bindings.py of the reference, the parts that need no
device), and the lattice generator against the reference's own."""
import json
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


def _read_vtk(path):
    """(n, points, velocity, {scalar name: values}) of a legacy binary VTK polydata file."""
    raw = path.read_bytes()
    assert raw.startswith(b"# vtk DataFile Version 3.0\nCryoSPH-CUDA particles\nBINARY\nDATASET POLYDATA\n")
    at = raw.index(b"POINTS ")
    n = int(raw[at:raw.index(b"\n", at)].split()[1])

    def block(tag, words, start):
        i = raw.index(tag, start)
        j = raw.index(b"\n", i) + 1
        return np.frombuffer(raw[j:j + 4 * words], dtype=">f4" if tag != b"VERTICES" else ">i4"), j + 4 * words

    pts, at = block(b"POINTS", 3 * n, 0)
    verts, at = block(b"VERTICES", 2 * n, at)
    scal = {}
    for name in (b"temperature", b"mass", b"density", b"phase", b"pressure"):
        if raw.find(b"SCALARS " + name, at) < 0:
            continue
        i = raw.index(b"LOOKUP_TABLE default\n", raw.index(b"SCALARS " + name, at)) + len(b"LOOKUP_TABLE default\n")
        scal[name.decode()] = np.frombuffer(raw[i:i + 4 * n], dtype=">f4")
        at = i + 4 * n
    vel, at = block(b"VECTORS velocity", 3 * n, at)
    assert raw[at:] == b"\n"
    assert np.array_equal(verts.reshape(n, 2)[:, 0], np.ones(n)) and np.array_equal(verts.reshape(n, 2)[:, 1],
                                                                                    np.arange(n))
    return n, pts.reshape(n, 3), vel.reshape(n, 3), scal


def test_vtk_writer_header_and_payload(tmp_path):
    """io test VtkHeaderAndSize (tests/test_io.cpp:21-32 of the reference),
    plus every value read back from the binary payload."""
    p = cs.make_block((0, 0, 0), (0.03, 0.02, 0.01), 0.01, cs.Phase.Liquid, 70.8, 20.3)
    assert len(p["mass"]) == 6
    p["velocity"] = np.arange(18, dtype=np.float32).reshape(6, 3) * 0.5
    path = tmp_path / "block.vtk"
    cs.write_vtk(str(path), p, np.full(6, 1e5))
    text = path.read_bytes()
    assert b"POINTS 6 float" in text and b"SCALARS pressure float 1" in text and b"VECTORS velocity float" in text
    n, pts, vel, scal = _read_vtk(path)
    assert n == 6
    assert np.array_equal(pts, p["position"].astype(np.float32))
    assert np.array_equal(vel, p["velocity"])
    assert np.array_equal(scal["temperature"], p["temperature"]) and np.array_equal(scal["mass"], p["mass"])
    assert np.array_equal(scal["density"], p["density"]) and np.array_equal(scal["phase"], np.zeros(6))
    assert np.array_equal(scal["pressure"], np.full(6, 1e5, np.float32))
    cs.write_vtk(str(path), p)  # no pressure: the section is left out
    _, _, _, scal = _read_vtk(path)
    assert "pressure" not in scal


def test_json_frame_filters_walls(tmp_path):
    """io test JsonFrameFiltersWalls (tests/test_io.cpp:34-46 of the reference)."""
    p = cs.make_block((0, 0, 0), (0.02, 0.01, 0.01), 0.01, cs.Phase.Liquid, 1000.0, 300.0)
    wall = {"position": [[1, 1, 1]], "mass": [1.0], "density": [1000.0], "temperature": [300.0], "phase": [2]}
    both = {k: np.concatenate([np.asarray(p[k]), np.asarray(wall[k], dtype=np.asarray(p[k]).dtype)])
            for k in wall}
    fr = cs.make_frame(both, None, 0.5, 42)
    path = tmp_path / "frame.json"
    cs.write_json_frame(str(path), fr, include_walls=False)
    s = path.read_text()
    assert '"step":42' in s and '"n":2' in s and '"phase":[0,0]' in s and '"temperature":[300,300]' in s
    d = json.loads(s)
    assert d["time"] == 0.5 and len(d["position"]) == 6 and d["pressure"] == [0, 0]
    cs.write_json_frame(str(path), fr, include_walls=True)
    d = json.loads(path.read_text())
    assert d["n"] == 3 and d["phase"] == [0, 0, 2] and d["position"][-3:] == [1, 1, 1]


def test_json_numbers_use_six_significant_digits(tmp_path):
    rng = np.random.default_rng(5)
    n = 200
    x = (rng.standard_normal((n, 3)) * 10.0 ** rng.integers(-8, 8, (n, 1))).astype(np.float32)
    T = (rng.random(n) * 400).astype(np.float32)
    T[3] = np.nan  # non-finite values are written as 0
    parts = {"position": x, "mass": np.ones(n), "density": np.ones(n), "temperature": T,
             "phase": np.zeros(n, np.uint8), "velocity": rng.standard_normal((n, 3))}
    fr = cs.make_frame(parts, np.linspace(-1e5, 1e5, n), 1.0 / 3.0, 7)
    path = tmp_path / "f.json"
    cs.write_json_frame(str(path), fr)
    d = json.loads(path.read_text())
    assert d["time"] == float("%.9g" % (1.0 / 3.0))
    assert d["position"] == [float("%.6g" % v) for v in x.ravel().astype(np.float64)]
    assert d["temperature"][3] == 0 and d["temperature"][4] == float("%.6g" % float(T[4]))
    speed = np.linalg.norm(np.asarray(parts["velocity"], np.float32), axis=1)
    assert np.allclose(d["speed"], speed, rtol=1e-5)


def test_particle_columns_reject_bad_shapes():
    ln2 = cs.FluidProperties.liquid_nitrogen()
    p = cs.make_block((0, 0, 0), (0.02, 0.01, 0.01), 0.01, cs.Phase.Liquid, 1000.0, 300.0)
    with pytest.raises(ValueError):
        cs.write_vtk("/dev/null", dict(p, mass=p["mass"][:-1]))
    with pytest.raises(ValueError):
        cs.write_vtk("/dev/null", dict(p, phase=np.full(len(p["mass"]), 7, np.uint8)))
    with pytest.raises(ValueError):
        cs.write_vtk("/dev/null", dict(p, position=p["position"][:, :2]))
    assert ln2.T_sat > 0


def test_mesh_tank_generator_matches_the_analytic_box(tmp_path):
    """A closed triangle mesh of a box fills like the analytic BoxTank: the same
    lattice nodes classified the same way (mesh distances from the
    point-triangle query, the sign from the winding number)."""
    verts = [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1)]
    faces = [(1, 3, 2), (1, 4, 3), (5, 6, 7), (5, 7, 8), (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6),
             (3, 4, 8), (3, 8, 7), (4, 1, 5), (4, 5, 8)]
    path = tmp_path / "box.obj"
    path.write_text("# a cube\n" + "".join(f"v {a} {b} {c}\n" for a, b, c in verts) +
                    "".join(f"f {a}/1/1 {b}/2/2 {c}/3/3\n" for a, b, c in faces))
    mesh = cs.MeshTank(str(path), scale=0.02)
    box = cs.BoxTank(0.04, 0.04, 0.04)
    ln2 = cs.FluidProperties.liquid_nitrogen()
    fill = cs.FillSpec()
    fill.fill_fraction = 0.4
    a = cs.tank_particles(mesh, ln2, 0.004, fill)
    b = cs.tank_particles(box, ln2, 0.004, fill)
    for k in ("position", "phase", "mass", "temperature", "flags", "id"):
        assert np.array_equal(a[k], b[k]), k
    assert np.allclose(a["normal"], b["normal"], atol=1e-6)
    assert mesh.volume() == pytest.approx(box.volume())


def test_obj_reader_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n")
    with pytest.raises(Exception):
        cs.MeshTank(str(p))
    p.write_text("v 0 0 0\nv 1 0 0\n")
    with pytest.raises(Exception):
        cs.MeshTank(str(p))
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf -4 -3 -2 -1\n")  # a quad by relative indices, fanned
    assert cs.MeshTank(str(p)).num_triangles == 2


def test_jitter_offsets_are_a_function_of_seed_and_id():
    """The host restatement of the device jitter: bounded by the amplitude,
    fixed by (seed, id, axis) whatever the order, different for another seed,
    and 24-bit uniform draws (mean near 0, variance near amp^2 / 3)."""
    ids = np.arange(200_000, dtype=np.uint32)
    a = cabi.jitter_offsets(ids, 2002, 1e-4)
    assert a.shape == (len(ids), 3) and a.dtype == np.float32
    assert np.abs(a).max() <= 1e-4
    perm = np.random.default_rng(1).permutation(len(ids))
    assert np.array_equal(cabi.jitter_offsets(ids[perm], 2002, 1e-4), a[perm])
    assert not np.array_equal(cabi.jitter_offsets(ids, 2003, 1e-4), a)
    assert abs(float(a.mean())) < 2e-7
    assert abs(float(a.var()) / (1e-4 ** 2 / 3.0) - 1.0) < 0.01
    # the three axes are not copies of one another
    assert abs(float(np.corrcoef(a[:, 0], a[:, 1])[0, 1])) < 0.01
