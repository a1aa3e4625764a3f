"""Parity of the CUDA path with the oracle at the benchmarked sizes and on the
paths the short scenarios do not reach.

* The dam break at the bench's lattice (dx 0.02 m, 203 662 particles): keys,
  permutation, cell tables and every neighbour list bit-exact; 5 steps with
  fields within 1e-5 (normwise), the FP64 diagnostics including the slosh
  force / moment, kinetic energy, centre of mass and momentum, and the
  probe pressures at the eight SPHERIC Test 2 sensors
  (validation/spheric_test2/run.py:69-73 of the reference).
* C1 as specified: relax 0.05 s, then 200 steps; fields, diagnostics and the
  neighbour lists of the final state against the oracle, with the FP32 noise
  floor of the trajectory measured against the reference's FP64 build.
* Splits and merges inside the window: heavy particles split
  (phase_change.cu:270-335 -- mark, scan, split with the hashed direction)
  and light vapour particles merge and die, so the next build gives them the
  dead sentinel key and compacts them away (spatial_hash.cu:61-68); ids,
  phases, counts and fields against the oracle.

Tolerances: integer and index results bit-exact; fields 1e-5 normwise
relative; FP64 diagnostics 1e-6 relative; float diagnostics (slosh force,
centre of mass, momentum: FP64 sums cast to float) 1e-5 relative to the
vector's magnitude.
"""
import numpy as np
import pytest

import cryo_cabi as cabi
import refpy
import scenarios as S

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-5
DIAG_RTOL = 1e-6
PERSISTENT = ["x", "v", "vt", "nrm", "m", "m0", "rho", "T", "phase", "flags", "id"]
STEP_FIELDS = ["x", "v", "m", "rho", "T", "p", "sigma", "a", "ab"]
FP64_DIAG = ["mass_liquid", "mass_vapor", "mass_total", "kinetic_energy", "enthalpy", "heat_input", "T_sat",
             "p_ullage", "evaporated_mass", "condensed_mass", "max_speed", "T_liquid_mean", "T_liquid_max",
             "T_vapor_mean", "time", "dt"]
VEC_DIAG = ["slosh_force", "slosh_moment", "liquid_com", "liquid_momentum"]
INT_DIAG = ["step", "n_total", "n_liquid", "n_vapor", "n_wall", "splits", "merges"]

# SPHERIC Test 2 pressure sensors: four on the obstacle's front face, four on
# its top, in the plane y = 0.403 / 2 - 0.176 (run.py:30-33, 69-73)
X_FRONT, BOX_H, SENSOR_Y = 0.744, 0.161, 0.403 / 2 - 0.176
OFFS = (0.021, 0.061, 0.101, 0.141)


def sensors(dx):
    front = [(X_FRONT + 0.5 * dx, SENSOR_Y, z) for z in OFFS]
    top = [(X_FRONT - o, SENSOR_Y, BOX_H + 0.5 * dx) for o in OFFS]
    return np.array(front + top, np.float32)


def pair(cfg, fl, parts, lo, hi):
    g = cabi.Context(cfg, fl)
    o = refpy.Oracle(cfg, fl)
    g.set_particles(parts, lo, hi)
    o.set_particles(parts, lo, hi)
    return g, o


def assert_grid_bit_exact(g, o):
    g.run_pass("grid_build")
    o.run_pass("grid_build")
    keys, perm, cs, ce = g.grid_tables()
    ok, op = o.grid_sort()
    ocs, oce = o.cell_tables()
    assert np.array_equal(keys, ok[: len(keys)]), "sorted keys differ"
    assert np.array_equal(perm, op[: len(perm)]), "permutation differs (stable sort)"
    assert np.array_equal(cs, ocs) and np.array_equal(ce, oce), "cell_start/cell_end differ"
    for f in PERSISTENT:
        assert np.array_equal(g.field(f).view(np.uint8), o.field(f).view(np.uint8)), f"{f} differs after reorder"
    gc, gl = g.neighbor_lists()
    oc, ol = o.neighbor_lists()
    assert np.array_equal(gc, oc), "neighbour counts differ"
    assert np.array_equal(gl, ol), "neighbour lists differ (membership or order)"
    S.assert_stored_lists(g, oc, ol, o.field("phase"))
    return len(gl)


def assert_fields(g, o, fields=STEP_FIELDS, tol=FIELD_RTOL, tag=""):
    worst = []
    for f in fields:
        err = S.normwise(g.field(f), o.field(f))
        worst.append((f, err))
        assert err <= tol, f"{tag} {f}: normwise error {err:.3e} > {tol:.1e}"
    for f in ["phase", "id"]:
        assert np.array_equal(g.field(f), o.field(f)), f"{tag} {f} differs"
    return worst


def assert_diagnostics(g, o, tag="", skip=()):
    dg, do = g.diagnostics().as_dict(), o.diagnostics().as_dict()
    for k in INT_DIAG:
        assert dg[k] == do[k], (tag, k, dg[k], do[k])
    for k in FP64_DIAG:
        ref = do[k]
        assert abs(dg[k] - ref) <= DIAG_RTOL * max(abs(ref), 1e-30) + 1e-30, (tag, k, dg[k], ref)
    for k in VEC_DIAG:
        if k in skip:
            continue
        a, b = np.asarray(dg[k], np.float64), np.asarray(do[k], np.float64)
        scale = max(float(np.linalg.norm(b)), 1e-30)
        assert float(np.abs(a - b).max()) <= FIELD_RTOL * scale, (tag, k, dg[k], do[k])
    return dg


def test_dam_break_at_bench_size_grid_and_lists_bit_exact(cuda_device):
    cfg, fl, parts, lo, hi = S.dam_break(dx=0.02)
    assert len(parts["x"]) == 203662
    g, o = pair(cfg, fl, parts, lo, hi)
    entries = assert_grid_bit_exact(g, o)
    print(f"\n[dam break dx 0.02] {len(parts['x'])} particles, {entries} list entries bit-exact")


def test_dam_break_at_bench_size_steps_diagnostics_and_probes(cuda_device):
    cfg, fl, parts, lo, hi = S.dam_break(dx=0.02)
    g, o = pair(cfg, fl, parts, lo, hi)
    pts = sensors(0.02)
    for k in range(5):
        g.step(1)
        o.step(1)
        assert_diagnostics(g, o, f"step {k + 1}")
        pg, po = g.probe_pressure(pts), o.probe_pressure(pts)
        assert np.array_equal(np.isnan(pg), np.isnan(po)), (k, pg, po)
        wet = ~np.isnan(po)
        if wet.any():
            assert S.normwise(pg[wet], po[wet]) <= FIELD_RTOL, (k, pg, po)
    worst = assert_fields(g, o, tag="dam break dx 0.02, 5 steps")
    # the dry sensors read NaN on both sides; the ones under the column read a pressure
    assert g.time()[0] == o.time()[0]
    print("\n[dam break dx 0.02] 5 steps, worst fields:", sorted(worst, key=lambda t: -t[1])[:3])


def test_dam_break_probe_series_on_wet_points(cuda_device):
    """Probe pressures where the column stands (a grid of points inside the
    water), every step of a short run: same NaN pattern and values."""
    cfg, fl, parts, lo, hi = S.dam_break(dx=0.04)
    g, o = pair(cfg, fl, parts, lo, hi)
    xs = np.linspace(3.22 - 1.2, 3.2, 6)
    zs = np.linspace(0.02, 0.6, 5)
    pts = np.array([(x, y, z) for x in xs for y in (-0.3, 0.0, 0.3) for z in zs], np.float32)
    for k in range(4):
        g.step(1)
        o.step(1)
        pg, po = g.probe_pressure(pts), o.probe_pressure(pts)
        assert np.array_equal(np.isnan(pg), np.isnan(po)), k
        wet = ~np.isnan(po)
        assert wet.sum() > len(pts) // 3
        assert S.normwise(pg[wet], po[wet]) <= FIELD_RTOL, k


def _by_id(ctx, f):
    order = np.argsort(ctx.field("id"), kind="stable")
    return ctx.field(f)[order].astype(np.float64)


@pytest.mark.skipif(not refpy.ref_available(fp64=True), reason="FP64 reference build (oracle/_ref) not present")
def test_c1_relax_then_200_steps(cuda_device):
    """C1 exactly as specified: relax(0.05) then 200 steps from the seeded
    lattice.  After the relax (about 20 steps) every field is within 1e-5 of
    the oracle.  Over the 200 steps the two FP32 runs separate slowly: both
    run the same IEEE operation sequence except single-precision libm calls
    (powf in the transport-velocity wall volume), which the C library rounds
    differently in the last bit for a small fraction of arguments.  The bar
    for the 200-step state is therefore the FP32 noise floor of this very
    trajectory, measured live: the oracle's own distance from the reference's
    FP64 build (particles aligned by id).  Every field of the CUDA run must be
    at least as close to the oracle as that, and no further from the FP64
    run than twice it.  The neighbour lists of the final state are compared
    bit for bit from the oracle's state on both sides."""
    cfg, fl, parts, lo, hi = S.c1()
    g, o = pair(cfg, fl, parts, lo, hi)
    r64 = refpy.Ref(cfg, fl, fp64=True)
    r64.set_threads(16)
    r64.set_particles(parts, lo, hi)
    g.relax(0.05)
    o.relax(0.05)
    r64.relax(0.05)
    assert_fields(g, o, ["x", "v", "m", "rho", "T"], tag="C1 after relax")
    g.step(200)
    o.step(200)
    r64.step(200)
    tg, sg, _ = g.time()
    to, so, _ = o.time()
    assert sg == so == 200 and abs(tg - to) <= 1e-6 * to
    for f in ["phase", "id"]:
        assert np.array_equal(g.field(f), o.field(f)), f
    report = []
    for f in ["x", "v", "m", "rho", "T", "p"]:
        floor = S.normwise(_by_id(o, f), _by_id(r64, f))
        vs_oracle = S.normwise(g.field(f), o.field(f))
        vs_fp64 = S.normwise(_by_id(g, f), _by_id(r64, f))
        report.append((f, vs_oracle, vs_fp64, floor))
        assert vs_oracle <= max(floor, FIELD_RTOL), (f, vs_oracle, floor)
        assert vs_fp64 <= 2.0 * floor + FIELD_RTOL, (f, vs_fp64, floor)
    dg, do, d64 = g.diagnostics().as_dict(), o.diagnostics().as_dict(), r64.diagnostics().as_dict()
    for k in INT_DIAG:
        assert dg[k] == do[k], (k, dg[k], do[k])
    for k in FP64_DIAG:
        tol = max(DIAG_RTOL * abs(do[k]), 2.0 * abs(do[k] - d64[k]), 1e-30)
        assert abs(dg[k] - do[k]) <= tol, (k, dg[k], do[k], d64[k])
    for k in VEC_DIAG:
        a, b, c = (np.asarray(d[k], np.float64) for d in (dg, do, d64))
        tol = max(FIELD_RTOL * float(np.linalg.norm(b)), 2.0 * float(np.abs(b - c).max()), 1e-30)
        assert float(np.abs(a - b).max()) <= tol, (k, dg[k], do[k], d64[k])
    # lists of the final state: the oracle's state on both sides, then the build
    for f in ["x", "v", "vt", "nrm", "m", "m0", "rho", "T"]:
        g.set_field(f, o.field(f))
    assert_grid_bit_exact(g, o)
    print("\n[C1 relax 0.05 + 200 steps] (field, vs oracle, vs FP64, oracle vs FP64):",
          [(f, f"{a:.2e}", f"{b:.2e}", f"{c:.2e}") for f, a, b, c in report])


def split_case():
    """LN2 boil-off cylinder with a split ratio of 1.02 and Lee 200 1/s:
    evaporation makes vapour particles heavy enough to split in step 1."""
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    cfg.update(split_ratio=1.02, lee_evaporation=200.0)
    return cfg, fl, parts, lo, hi


def merge_case():
    """Subcooled LN2 cylinder with strong condensation and a merge ratio of
    0.98: vapour particles condense below the ratio, merge into liquid
    neighbours and die in step 1; the next build compacts them away."""
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1, lee_evaporation=0.0,
                         lee_condensation=400.0, merge_ratio=0.98, heater_power=0.0, velocity_scale=1)
    parts, lo, hi = S.tank([(refpy.CYLINDER, 0, 0, (0.03, 0.075, 0))], fl, 0.004,
                           refpy.make_fill(fill_fraction=0.5, T_liquid=fl.T_sat - 3, T_vapor=fl.T_sat - 2))
    return cfg, fl, parts, lo, hi


@pytest.mark.parametrize("name,mk", [("split", split_case), ("merge", merge_case)])
def test_split_and_merge_match_the_oracle(cuda_device, name, mk):
    cfg, fl, parts, lo, hi = mk()
    g, o = pair(cfg, fl, parts, lo, hi)
    n0 = len(parts["x"])
    g.step(1)
    o.step(1)
    # a step that splits sums the wall force of the new halves' slots, which no
    # force pass wrote (the reference leaves them as memory held them): the
    # slosh sums are compared where nothing split
    skip = ("slosh_force", "slosh_moment") if name == "split" else ()
    dg = assert_diagnostics(g, o, f"{name} step 1", skip=skip)
    assert g.num_particles() == o.num_particles()
    if name == "split":
        assert dg["splits"] > 0 and g.num_particles() == n0 + dg["splits"]
        # the children take ids next_id + k in slot order (phase_change.cu:320-335)
        assert np.array_equal(g.field("id"), o.field("id"))
    else:
        assert dg["merges"] > 0
        dead_g, dead_o = g.field("phase") == 3, o.field("phase") == 3
        assert dead_o.sum() == dg["merges"] and np.array_equal(dead_g, dead_o)
    assert_fields(g, o, ["x", "v", "m", "rho", "T"], tag=f"{name} step 1")
    # the next build sorts the dead to the end (sentinel key = num_cells) and
    # drops them; from the oracle's state on both sides (a split child's
    # position comes from cbrtf / cosf / sinf, which the C library and the
    # device round differently in the last bit for some arguments)
    for f in ["x", "v", "vt", "nrm", "m", "m0", "rho", "T"]:
        g.set_field(f, o.field(f))
    assert_grid_bit_exact(g, o)
    if name == "merge":
        assert g.num_particles() == n0 - dg["merges"]
    g2, o2 = pair(cfg, fl, parts, lo, hi)
    g2.step(4)
    o2.step(4)
    assert g2.num_particles() == o2.num_particles()
    if name == "merge":
        assert g2.num_particles() == n0 - dg["merges"], "the dead were compacted away"
        assert not (g2.field("phase") == 3).any()
    assert_fields(g2, o2, tag=f"{name} 4 steps")
    assert_diagnostics(g2, o2, f"{name} 4 steps", skip=skip)
