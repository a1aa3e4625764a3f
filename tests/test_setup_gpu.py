"""The tank lattice generated on the GPU (cryo_build_tank, through
Solver.build_tank) against the host generator (build_tank_particles,
geometry.cpp:242-330, itself bit-identical to the reference's): every particle
array equal bit for bit, for each primitive, CSG trees, every fill mode, the
heater band, vapour left out, and the extreme fill fractions."""
import time

import numpy as np
import pytest

import CryoSPH as cs

pytestmark = pytest.mark.gpu


def fill(mode=cs.FillMode.Settled, frac=0.5, **kw):
    f = cs.FillSpec()
    f.mode = mode
    f.fill_fraction = frac
    for k, v in kw.items():
        setattr(f, k, v)
    return f


def dam_break_geometry():
    tank = cs.Translated(cs.BoxTank(3.22, 1.0, 1.0), (1.61, 0.0, 0.5))
    box = (0.161, 0.403, 0.161)
    obst = cs.Translated(cs.BoxTank(*box), (0.744 - box[0] / 2, 0.0, box[2] / 2))
    return cs.Difference(tank, obst)


CASES = {
    "box_settled": (lambda: cs.BoxTank(0.04, 0.05, 0.03), lambda: fill(), 0.002),
    "cylinder_tilted": (lambda: cs.CylinderTank(0.05, 0.12), lambda: fill(frac=0.37, settle_direction=(0.3, -0.2, -1.0)),
                        0.004),
    "sphere_bubble": (lambda: cs.SphereTank(0.05), lambda: fill(cs.FillMode.CentralBubble, 0.8,
                                                                  bubble_center=(0.0, 0.01, -0.005)), 0.004),
    "capsule_no_vapour": (lambda: cs.CapsuleTank(0.02, 0.03), lambda: fill(frac=0.6, include_vapor=False), 0.002),
    "dam_break_full": (dam_break_geometry, lambda: fill(cs.FillMode.Full), 0.04),
    "union_heater": (lambda: cs.Union(cs.CylinderTank(0.03, 0.06), cs.Translated(cs.SphereTank(0.025), (0.0, 0.0, 0.04))),
                     lambda: fill(frac=0.5, heater_zmin=-0.01, heater_zmax=0.02, wall_layers=4, T_liquid=80.0,
                                  T_wall=90.0), 0.003),
    "all_vapour": (lambda: cs.BoxTank(0.03, 0.03, 0.03), lambda: fill(frac=0.0), 0.003),
    "all_liquid_settled": (lambda: cs.BoxTank(0.03, 0.03, 0.03), lambda: fill(frac=1.0), 0.003),
}


def build(geo, f, dx, on_device):
    cfg = cs.SolverConfig()
    cfg.dx = dx
    s = cs.Solver(cfg, cs.FluidProperties.liquid_nitrogen())
    s.build_tank(geo, f, on_device=on_device)
    return s


@pytest.mark.parametrize("name", sorted(CASES))
def test_device_lattice_equals_host_lattice(cuda_device, name):
    make_geo, make_fill, dx = CASES[name]
    dev = build(make_geo(), make_fill(), dx, True)
    host = build(make_geo(), make_fill(), dx, False)
    assert dev.num_particles == host.num_particles > 0
    pd, ph = dev.particles(), host.particles()
    for k in pd:
        a, b = np.asarray(pd[k]), np.asarray(ph[k])
        assert a.shape == b.shape, k
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    # and both equal the host generator's own arrays
    ref = cs.tank_particles(make_geo(), cs.FluidProperties.liquid_nitrogen(), dx, make_fill())
    assert np.array_equal(pd["position"], ref["position"].astype(pd["position"].dtype))
    assert np.array_equal(pd["phase"], ref["phase"])


def test_device_lattice_steps_like_host_lattice(cuda_device):
    """A tank built either way steps to the same state."""
    make_geo, make_fill, dx = CASES["cylinder_tilted"]
    dev, host = build(make_geo(), make_fill(), dx, True), build(make_geo(), make_fill(), dx, False)
    dev.run_steps(5)
    host.run_steps(5)
    assert dev.diagnostics().as_dict() == host.diagnostics().as_dict()


def test_device_lattice_timing_large_sphere(cuda_device):
    """The LH2 sphere workload (R 0.5 m, dx 5.2 mm, ~4 M particles), both ways."""
    geo, f, dx = cs.SphereTank(0.5), fill(), 0.0052
    t0 = time.perf_counter()
    dev = build(geo, f, dx, True)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    host = build(geo, f, dx, False)
    t_host = time.perf_counter() - t0
    print(f"\n[setup] {dev.num_particles} particles: device {t_dev:.3f} s, host {t_host:.3f} s (incl. upload)")
    assert dev.num_particles == host.num_particles
    for k in ("position", "phase", "normal"):
        assert np.array_equal(np.asarray(dev.particles()[k]), np.asarray(host.particles()[k])), k


def test_device_jitter_equals_its_host_restatement(cuda_device):
    """Solver.jitter_fluid moves the fluid lattice on the device; the same
    offsets from cryo_cabi.jitter_offsets (by particle id) applied to the host
    generator's particles give the same positions bit for bit; walls stay."""
    import cryo_cabi as cabi
    ln2 = cs.FluidProperties.liquid_nitrogen()
    cfg = cs.SolverConfig()
    cfg.dx = 0.004
    fill = cs.FillSpec()
    fill.fill_fraction = 0.4
    geo = cs.SphereTank(0.05)
    s = cs.Solver(cfg, ln2)
    s.build_tank(geo, fill)
    amp, seed = 0.05 * 0.004, 2002
    s.jitter_fluid(amp, seed)
    got = s.particles()
    host = cs.tank_particles(geo, ln2, 0.004, fill)
    off = cabi.jitter_offsets(host["id"], seed, amp)
    fl = host["phase"] != 2
    want = host["position"].astype(np.float32).copy()
    want[fl] = want[fl] + off[fl]
    order = np.argsort(got["id"])
    assert np.array_equal(got["id"][order], host["id"])
    assert np.array_equal(got["position"][order].view(np.uint32), want.view(np.uint32))
    assert np.abs(off).max() <= amp and off[fl].std() > 0.4 * amp
    s.run_steps(1)
    with pytest.raises(ValueError):
        s.jitter_fluid(amp, seed)
