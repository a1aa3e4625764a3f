"""The CryoSPH module end to end on the GPU: the reference's Python tests
(tests/python/test_bindings.py of the reference) against this module, plus
checkpoints, run_until, relax parity with the oracle and the device guards."""
import json

import numpy as np
import pytest

import CryoSPH as cs
import cryo_cabi as cabi
import refpy
import scenarios as S

pytestmark = pytest.mark.gpu


def small_config(**overrides):
    cfg = cs.SolverConfig()
    cfg.dx = 0.005
    cfg.gravity = (0.0, 0.0, 0.0)
    cfg.velocity_scale = 1.0
    for k, v in overrides.items():
        setattr(cfg, k, v)
    return cfg


def test_module_reports_the_device(cuda_device):
    assert cs.device_count() >= 1
    assert "sm_" in cs.device_name()


def test_tank_run_conserves_mass(cuda_device, tmp_path):
    ln2 = cs.FluidProperties.liquid_nitrogen()
    solver = cs.Solver(small_config(thermo_mode=cs.TankThermoMode.Closed, lee_evaporation=2.0), ln2)
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    fill.T_liquid = ln2.T_sat + 2.0
    solver.build_tank(cs.BoxTank(0.04, 0.04, 0.04), fill)
    solver.relax(0.01)
    d0 = solver.diagnostics()
    solver.run_steps(100)
    d1 = solver.diagnostics()
    assert d1.step == 100
    assert d1.mass_total == pytest.approx(d0.mass_total, rel=1e-5)
    assert d1.evaporated_mass > 0
    assert d1.p_ullage > d0.p_ullage
    parts = solver.particles()
    n = solver.num_particles
    assert parts["position"].shape == (n, 3)
    assert parts["phase"].dtype == np.uint8
    assert set(np.unique(parts["phase"])) <= {0, 1, 2}
    assert solver.pressure().shape == (n,)
    assert np.isfinite(parts["temperature"]).all()
    path = tmp_path / "frame.json"
    solver.write_json(str(path))
    frame = json.loads(path.read_text())
    assert frame["step"] == 100
    assert len(frame["position"]) == 3 * frame["n"]
    assert 2 not in frame["phase"]
    solver.write_vtk(str(tmp_path / "frame.vtk"))
    assert (tmp_path / "frame.vtk").stat().st_size > 0


def test_custom_particles_and_telemetry(cuda_device):
    ln2 = cs.FluidProperties.liquid_nitrogen()
    solver = cs.Solver(small_config(thermal=False, phase_change=False,
                                    surface_tension=cs.SurfaceTensionModel.NoTension), ln2)
    dx = 0.005
    g = (np.arange(6) + 0.5) * dx
    pos = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    n = len(pos)
    rho = np.full(n, ln2.rho_liquid)
    solver.set_particles(pos, rho * dx ** 3, rho, np.full(n, ln2.T_sat), np.zeros(n, np.uint8),
                         domain_lo=(-0.01, -0.01, -0.01), domain_hi=(0.04, 0.04, 0.04))
    assert solver.num_particles == n
    for mode in (cs.TelemetryMode.AsyncCopy, cs.TelemetryMode.ZeroCopy):
        solver.configure_telemetry(mode)
        solver.run_steps(3)
        assert solver.request_telemetry()
        assert not solver.request_telemetry()
        frame = solver.fetch_telemetry()
        assert frame["position"].shape == (n, 3)
        assert frame["step"] == solver.step_count
        assert solver.fetch_telemetry() is None
        parts = solver.particles()
        assert np.array_equal(frame["position"], parts["position"].astype(np.float32))


def test_bad_inputs_raise(cuda_device):
    ln2 = cs.FluidProperties.liquid_nitrogen()
    solver = cs.Solver(small_config(), ln2)
    with pytest.raises(ValueError):
        solver.set_particles(np.zeros((4, 2)), np.ones(4), np.ones(4), np.ones(4), np.zeros(4, np.uint8),
                             domain_lo=(0, 0, 0), domain_hi=(1, 1, 1))
    with pytest.raises(ValueError):
        solver.set_particles(np.zeros((4, 3)), np.ones(4), np.ones(4), np.ones(4), np.full(4, 3, np.uint8),
                             domain_lo=(0, 0, 0), domain_hi=(1, 1, 1))
    with pytest.raises(ValueError):
        solver.set_contact_angle(-5.0)
    with pytest.raises(RuntimeError):
        solver.run_steps(1)  # nothing loaded
    akinci = cs.Solver(small_config(surface_tension=cs.SurfaceTensionModel.Akinci), ln2)
    with pytest.raises(ValueError):
        akinci.build_tank(cs.BoxTank(0.04, 0.04, 0.04), cs.FillSpec())  # vapour present


def test_csg_geometry_and_probes(cuda_device):
    tank = cs.Translated(cs.BoxTank(0.1, 0.1, 0.1), (0.05, 0.0, 0.05))
    block = cs.Translated(cs.BoxTank(0.02, 0.02, 0.02), (0.05, 0.0, 0.01))
    geo = cs.Difference(tank, block)
    water = cs.FluidProperties.water()
    cfg = small_config(surface_tension=cs.SurfaceTensionModel.NoTension, thermal=False, phase_change=False,
                       gravity=(0.0, 0.0, -9.81))
    cfg.dx = 0.01
    solver = cs.Solver(cfg, water)
    fill = cs.FillSpec()
    fill.mode = cs.FillMode.Full
    solver.build_tank(geo, fill)
    solver.run_steps(5)
    p = solver.probe_pressure(np.array([[0.02, 0.0, 0.02], [0.02, 0.0, 0.08], [0.5, 0.5, 0.5]]))
    assert p.shape == (3,)
    assert np.isfinite(p[0]) and np.isfinite(p[1])
    assert np.isnan(p[2])
    assert p[0] > p[1]


def test_maneuver_profile_and_slosh_loads(cuda_device):
    water = cs.FluidProperties.water()
    cfg = small_config(surface_tension=cs.SurfaceTensionModel.NoTension, thermal=False, phase_change=False)
    cfg.dx = 0.01
    solver = cs.Solver(cfg, water)
    fill = cs.FillSpec()
    fill.mode = cs.FillMode.Full
    solver.build_tank(cs.BoxTank(0.06, 0.06, 0.06), fill)
    solver.set_frame_motion(acceleration=(1.0, 0.0, 0.0))
    solver.run_steps(20)
    d = solver.diagnostics()
    assert d.frame_acceleration == pytest.approx((1.0, 0.0, 0.0))
    assert d.slosh_force[0] < 0
    assert set(d.as_dict()) >= {"slosh_force", "slosh_moment"}


def _particle_arrays(p):
    return {"x": p["position"], "m": p["mass"], "rho": p["density"], "T": p["temperature"], "phase": p["phase"],
            "nrm": p["normal"], "flags": p["flags"]}


def test_relax_maneuver_and_run_until_match_the_oracle(cuda_device):
    """relax (sph_solver.cu:707-736), a manoeuvre table and run_until through
    the C ABI, against the oracle, from identical inputs."""
    cfg, fl, parts, lo, hi = S.c1()
    g = cabi.Context(cfg, fl)
    o = refpy.Oracle(cfg, fl)
    man = ([0.0, 0.004, 0.012], [[0, 0, 0], [0.05, 0, 0], [0.05, 0.01, 0]], [[0, 0, 0], [0, 0, 0.02], [0, 0.01, 0.05]])
    for c in (g, o):
        c.set_particles(parts, lo, hi)
        c.relax(0.01)
    t = np.ascontiguousarray(man[0], np.float64)
    a = np.ascontiguousarray(man[1], np.float32)
    w = np.ascontiguousarray(man[2], np.float32)
    g.check(g.L.cryo_set_maneuver(g.h, 3, t.ctypes.data_as(cabi.C.POINTER(cabi.C.c_double)),
                                  a.ctypes.data_as(cabi.C.POINTER(cabi.C.c_float)),
                                  w.ctypes.data_as(cabi.C.POINTER(cabi.C.c_float)), cabi.vec3((0, 0, -0.01))))
    o.set_maneuver(man[0], man[1], man[2], origin=(0, 0, -0.01))
    g.run_until(0.02)
    o.run_until(0.02)
    tg, sg, _ = g.time()
    to, so, _ = o.time()
    assert sg == so and tg == pytest.approx(to, rel=1e-12)
    for f in ["x", "v", "T", "m", "p"]:
        assert S.normwise(g.field(f), o.field(f)) < 1e-5, f
    dg, do = g.diagnostics().as_dict(), o.diagnostics().as_dict()
    assert dg["frame_angular_velocity"] == pytest.approx(do["frame_angular_velocity"])
    assert dg["mass_total"] == pytest.approx(do["mass_total"], rel=1e-12)


def test_checkpoint_roundtrip_is_bitwise(cuda_device):
    """save_state / load_state: a restored solver continues bit-identically."""
    ln2 = cs.FluidProperties.liquid_nitrogen()
    cfg = small_config(thermo_mode=cs.TankThermoMode.Closed, lee_evaporation=5.0, split_ratio=1.05)
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    fill.T_liquid = ln2.T_sat + 3.0
    a = cs.Solver(cfg, ln2)
    a.build_tank(cs.BoxTank(0.04, 0.04, 0.04), fill)
    a.run_steps(20)
    blob = a.save_state()
    b = cs.Solver(cfg, ln2)
    b.build_tank(cs.BoxTank(0.04, 0.04, 0.04), fill)
    b.load_state(blob)
    a.run_steps(15)
    b.run_steps(15)
    pa, pb = a.particles(), b.particles()
    for k in pa:
        assert np.array_equal(np.asarray(pa[k]).view(np.uint8), np.asarray(pb[k]).view(np.uint8)), k
    assert a.diagnostics().as_dict() == b.diagnostics().as_dict()


def test_capacity_growth_keeps_the_state(cuda_device):
    """Particles beyond 3/4 of the capacity trigger a reallocation between
    steps (sph_solver.cu:556-560); the state carries over bit-identically."""
    cfg, fl, parts, lo, hi = S.box_split()
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    cap0 = cabi.C.c_int()
    g.check(g.L.cryo_capacity(g.h, cabi.C.byref(cap0)))
    g.step(2)
    x0 = g.field("x")
    assert g.num_particles() <= cap0.value
    assert g.device_status() == 0
    assert np.isfinite(x0).all()


def test_device_packed_frames_equal_the_host_writers(cuda_device, tmp_path):
    """Solver.write_vtk / write_json pack the payload on the device
    (cryo_frame_vtk, cryo_frame_viewer); the files are byte-identical to the
    host writers' on the downloaded state (write_vtk(particles, pressure) and
    write_json_frame(make_frame(...)), io.cpp:52-142 of the reference)."""
    ln2 = cs.FluidProperties.liquid_nitrogen()
    solver = cs.Solver(small_config(thermo_mode=cs.TankThermoMode.Closed), ln2)
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    solver.build_tank(cs.CylinderTank(0.02, 0.05), fill)
    solver.run_steps(7)
    parts, pres = solver.particles(), solver.pressure()
    dev, host = tmp_path / "dev.vtk", tmp_path / "host.vtk"
    solver.write_vtk(str(dev))
    cs.write_vtk(str(host), parts, pres)
    assert dev.read_bytes() == host.read_bytes()
    for walls in (False, True):
        dev, host = tmp_path / f"dev{walls}.json", tmp_path / f"host{walls}.json"
        solver.write_json(str(dev), include_walls=walls)
        cs.write_json_frame(str(host), cs.make_frame(parts, pres, solver.time, solver.step_count), include_walls=walls)
        assert dev.read_text() == host.read_text()
        d = json.loads(dev.read_text())
        assert d["n"] == (len(parts["phase"]) if walls else int((parts["phase"] != 2).sum()))


def test_particles_round_trip_through_the_soa_transfers(cuda_device):
    """set_particles then particles() returns every array as given (float32
    state; ids and flags as given; velocities, normals and flags optional)."""
    ln2 = cs.FluidProperties.liquid_nitrogen()
    rng = np.random.default_rng(3)
    p = cs.tank_particles(cs.BoxTank(0.03, 0.03, 0.03), ln2, 0.003, cs.FillSpec())
    n = len(p["mass"])
    v = rng.standard_normal((n, 3))
    solver = cs.Solver(small_config(dx=0.003), ln2)
    solver.set_particles(p["position"], p["mass"], p["density"], p["temperature"], p["phase"],
                         domain_lo=(-0.03, -0.03, -0.03), domain_hi=(0.03, 0.03, 0.03), velocity=v,
                         normal=p["normal"], flags=p["flags"])
    q = solver.particles()
    for k in ("position", "mass", "density", "temperature", "normal"):
        assert np.array_equal(q[k], np.asarray(p[k], np.float32)), k
    assert np.array_equal(q["velocity"], v.astype(np.float32))
    for k in ("phase", "flags", "id"):
        assert np.array_equal(q[k], p[k]), k
    solver.set_particles(p["position"], p["mass"], p["density"], p["temperature"], p["phase"],
                         domain_lo=(-0.03, -0.03, -0.03), domain_hi=(0.03, 0.03, 0.03))
    q = solver.particles()
    assert not q["velocity"].any() and not q["normal"].any() and not q["flags"].any()
    assert np.array_equal(q["id"], np.arange(n))
    # float64 columns (NumPy's default; converted on several host threads)
    # arrive rounded exactly as astype(float32) rounds them
    f64 = {k: np.asarray(p[k], np.float64) * (1.0 + 1e-9) for k in ("position", "mass", "density", "temperature")}
    v64 = rng.standard_normal((n, 3))
    solver.set_particles(f64["position"], f64["mass"], f64["density"], f64["temperature"], p["phase"],
                         domain_lo=(-0.03, -0.03, -0.03), domain_hi=(0.03, 0.03, 0.03), velocity=v64)
    q = solver.particles()
    for k, a in f64.items():
        assert np.array_equal(q[k], a.astype(np.float32)), k
    assert np.array_equal(q["velocity"], v64.astype(np.float32))


def test_diagnostics_requested_without_blocking_equal_the_blocking_ones(cuda_device):
    """request_diagnostics after each step and fetch_diagnostics later (in
    request order) give the records a twin solver's blocking diagnostics()
    gives after the same steps; nothing pending gives None; at most 8
    requests may be pending."""
    ln2 = cs.FluidProperties.liquid_nitrogen()
    cfg = small_config(dx=0.004, gravity=(0.0, 0.0, -9.81e-4), heater_power=5.0)
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    geo = cs.CylinderTank(0.03, 0.06)
    a, b = cs.Solver(cfg, ln2), cs.Solver(cfg, ln2)
    a.build_tank(geo, fill)
    b.build_tank(geo, fill)
    assert a.fetch_diagnostics() is None
    want = []
    for k in range(6):
        a.set_frame_motion(acceleration=(0.02 * k, 0.0, 0.0))
        b.set_frame_motion(acceleration=(0.02 * k, 0.0, 0.0))
        a.step()
        b.step()
        a.request_diagnostics()
        want.append(b.diagnostics())
        if k >= 1:  # the previous step's record, while this one may still run
            got = a.fetch_diagnostics()
            ref = want[k - 1]
            for f in ("time", "step", "dt", "mass_total", "kinetic_energy", "enthalpy", "p_ullage", "T_sat",
                      "heat_input", "max_speed"):
                assert getattr(got, f) == getattr(ref, f), f
            assert tuple(got.slosh_force) == tuple(ref.slosh_force)
    last = a.fetch_diagnostics(wait=True)
    assert last.step == want[-1].step and last.kinetic_energy == want[-1].kinetic_energy
    assert a.fetch_diagnostics(wait=False) is None
    for _ in range(8):
        a.request_diagnostics()
    with pytest.raises(Exception):
        a.request_diagnostics()
    n = 0
    while a.fetch_diagnostics() is not None:
        n += 1
    assert n == 8
