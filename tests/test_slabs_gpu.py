"""Slab decomposition of one tank (cryo_slabs_*): the tank cut along z into
slabs of cell layers, each a context of its own on the one device, with halo
layers copied between passes.  Its particles must equal, bit for bit and in
the same order, those of the one-context run over the same steps (the slabs'
sorted orders are the whole tank's, cut at layer boundaries); the FP64
diagnostics are added per slab and agree to rounding."""
import numpy as np
import pytest

import cryo_cabi as cabi
import scenarios as S

pytestmark = pytest.mark.gpu

FIELDS = ("x", "v", "T", "m", "rho", "phase", "flags", "id", "nrm")


def one_context(cfg, fl, parts, lo, hi, steps):
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    g.step(steps)
    out = {k: g.field(k) for k in FIELDS}
    return out, g.diagnostics(), g


def slabs(cfg, fl, parts, lo, hi, nslabs, steps):
    s = cabi.Slabs(cfg, fl, nslabs)
    s.set_particles(parts, lo, hi)
    s.step(steps)
    return s.particles(), s.diagnostics(), s


def assert_same(ref, got, what):
    for k in FIELDS:
        a, b = ref[k], got[k]
        assert a.shape == b.shape, f"{what}: {k} shape {a.shape} vs {b.shape}"
        if a.dtype.kind == "f":
            same = (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))
        else:
            same = a == b
        bad = np.flatnonzero(~same.reshape(len(a), -1).all(axis=1))
        assert bad.size == 0, f"{what}: {k} differs at {bad.size} particles, first {bad[:5]}"


def assert_diag_close(d1, d2, what, slosh=True):
    for f in ("time", "step", "dt", "n_total", "n_liquid", "n_vapor", "n_wall", "splits", "merges", "T_sat",
              "heat_input"):
        assert getattr(d1, f) == getattr(d2, f), f"{what}: {f} {getattr(d1, f)} vs {getattr(d2, f)}"
    for f in ("mass_liquid", "mass_vapor", "kinetic_energy", "enthalpy", "evaporated_mass", "condensed_mass",
              "p_ullage"):
        a, b = getattr(d1, f), getattr(d2, f)
        assert abs(a - b) <= 1e-12 * max(abs(a), abs(b), 1e-300), f"{what}: {f} {a} vs {b}"
    for k in range(3 if slosh else 0):
        a, b = d1.slosh_force[k], d2.slosh_force[k]
        assert abs(a - b) <= 1e-6 * max(abs(a), 1e-12), f"{what}: slosh_force[{k}] {a} vs {b}"


CASES = {
    "dam_break": lambda: S.dam_break(0.04),
    "c1": lambda: S.c1(),
    "ln2_boiloff": lambda: S.ln2_boiloff(),
    "lh2_sphere": lambda: S.lh2_sphere(),
    "options": lambda: S.options(),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("nslabs", [1, 2, 3])
def test_slabs_equal_one_context(cuda_device, name, nslabs):
    cfg, fl, parts, lo, hi = CASES[name]()
    steps = 12
    ref, d_ref, _ = one_context(cfg, fl, parts, lo, hi, steps)
    got, d_got, s = slabs(cfg, fl, parts, lo, hi, nslabs, steps)
    zb, owned, held = s.layout()
    print(f"\n[{name} x{nslabs}] layers {zb.tolist()} owned {owned.tolist()} held {held.tolist()}")
    assert owned.sum() == len(ref["x"])
    assert s.graph_mode() == 1, "the slab steps should replay the captured group graph"
    assert_same(ref, got, f"{name} x{nslabs}")
    assert_diag_close(d_ref, d_got, f"{name} x{nslabs}")


def test_slab_graph_and_host_threads_agree(cuda_device):
    """The captured group step (graph mode, the default) and the same steps
    enqueued by one host thread per slab meeting at barriers give the same
    particles bit for bit, with splits inside the window and steps issued in
    several calls (re-captures after capacity changes included)."""
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    cfg.update(split_ratio=1.02, lee_evaporation=200.0)
    runs = []
    for graph in (True, False):
        s = cabi.Slabs(cfg, fl, 3)
        s.set_graph_mode(graph)
        s.set_particles(parts, lo, hi)
        for k in (1, 7, 16, 6):
            s.step(k)
        assert s.graph_mode() == (1 if graph else 0)
        runs.append((s.particles(), s.diagnostics()))
    assert runs[0][1].splits > 0, "the case should split particles"
    assert_same(runs[1][0], runs[0][0], "graph vs host threads")
    assert_diag_close(runs[1][1], runs[0][1], "graph vs host threads")


def test_slabs_with_splits(cuda_device):
    """Heavy particles split inside the window: the new ids follow the slab
    order, as the one-context run's slot scan gives them."""
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    cfg.update(split_ratio=1.02, lee_evaporation=200.0)
    steps = 20
    ref, d_ref, _ = one_context(cfg, fl, parts, lo, hi, steps)
    assert d_ref.splits > 0, "the case should split particles"
    got, d_got, _ = slabs(cfg, fl, parts, lo, hi, 3, steps)
    assert_same(ref, got, "splits x3")
    # the slosh sums of a step that split particles include the new halves'
    # wall-force slots, which no force pass wrote (left in memory by earlier
    # particles in the one-context run, zero in the slabs)
    assert_diag_close(d_ref, d_got, "splits x3", slosh=False)


def test_slabs_run_in_batches(cuda_device):
    """Steps issued in several calls (the slabs check their guard words and
    head-room between calls) give the same state as one call."""
    cfg, fl, parts, lo, hi = S.c1()
    ref, _, _ = one_context(cfg, fl, parts, lo, hi, 40)
    s = cabi.Slabs(cfg, fl, 2)
    s.set_particles(parts, lo, hi)
    for k in (1, 7, 16, 16):
        s.step(k)
    assert_same(ref, s.particles(), "batches")


def test_slabs_reject_thin_tanks(cuda_device):
    cfg, fl, parts, lo, hi = S.options()
    s = cabi.Slabs(cfg, fl, 6)
    with pytest.raises(cabi.CryoError) as e:
        s.set_particles(parts, lo, hi)
    assert e.value.code == cabi.CRYO_EINVAL


def test_slab_solver_python_api(cuda_device):
    """CryoSPH.SlabSolver (the module API) against CryoSPH.Solver on a
    generated tank: the same particle dict after the same steps."""
    import CryoSPH as cs
    fluid = cs.FluidProperties.liquid_nitrogen()
    cfg = cs.SolverConfig()
    cfg.dx = 0.004
    cfg.gravity = (0.0, 0.0, -9.81e-4)
    cfg.heater_power = 20.0
    cfg.thermo_mode = cs.TankThermoMode.Closed
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    geo = cs.CylinderTank(0.05, 0.12)
    one = cs.Solver(cfg, fluid)
    one.build_tank(geo, fill, on_device=False)
    one.run_steps(10)
    sl = cs.SlabSolver(cfg, fluid, slabs=3)
    sl.build_tank(geo, fill)
    sl.run_steps(10)
    a, b = one.particles(), sl.particles()
    assert sl.num_particles == one.num_particles
    for k in a:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    lay = sl.layout()
    assert len(lay["z_begin"]) == 4 and sum(lay["owned"]) == one.num_particles
    assert sl.diagnostics().step == one.diagnostics().step == 10
    assert sl.graph_mode == 1
    sl.graph_mode = False
    assert sl.graph_mode == 0
