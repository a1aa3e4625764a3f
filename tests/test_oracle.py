"""The oracle (oracle/cryo_oracle.c) is the checker of the CUDA path; these
CPU tests pin it to the reference: bit for bit against the committed golden
vectors (made by tests/golden/make_golden.py from the reference's own CPU
build) and, where that build is present (oracle/_ref), live on several
scenarios including splits, venting, relax and a manoeuvre."""
import os

import numpy as np
import pytest

import cryo_cabi as cabi
import refpy
import scenarios as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
needs_ref = pytest.mark.skipif(not refpy.ref_available(), reason="reference CPU build (oracle/_ref) not built")


def same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def load_inputs(z):
    parts = {k[3:]: z[k] for k in z.files if k.startswith("in_") and k not in ("in_lo", "in_hi")}
    return parts, tuple(z["in_lo"]), tuple(z["in_hi"])


def test_oracle_matches_golden_box_split():
    z = np.load(os.path.join(GOLDEN, "box_split.npz"))
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -0.5), contact_angle_deg=10, velocity_scale=1, thermo_mode=1,
                         lee_evaporation=5, lee_condensation=5, split_ratio=1.05)
    parts, lo, hi = load_inputs(z)
    o = refpy.Oracle(cfg, fl)
    o.set_particles(parts, lo, hi)
    for tag, steps in (("s1", 1), ("s200", 199)):
        o.step(steps)
        for f in cabi.FIELDS:
            if tag == "s200" and f == "rmin":
                continue  # the reference leaves rmin of freshly split slots unset
            assert same_bits(o.field(f), z[f"{tag}_{f}"]), (tag, f)
        d = o.diagnostics().as_dict()
        for k in ["mass_total", "enthalpy", "p_ullage", "T_sat", "splits", "evaporated_mass", "time"]:
            assert d[k] == z[f"{tag}_diag_{k}"][()], (tag, k, d[k], z[f"{tag}_diag_{k}"])
    assert int(z["s200_diag_splits"]) > 0, "the golden scenario exercises splitting"


def test_oracle_matches_golden_grid_and_neighbors():
    z = np.load(os.path.join(GOLDEN, "c1_pass.npz"))
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), heater_power=20.0, thermo_mode=1)
    parts, lo, hi = load_inputs(z)
    o = refpy.Oracle(cfg, fl)
    o.set_particles(parts, lo, hi)
    o.run_pass("grid_build")
    cs, ce = o.cell_tables()
    assert np.array_equal(cs, z["cell_start"]) and np.array_equal(ce, z["cell_end"])
    assert np.array_equal(o.field("id"), z["sorted_id"])
    assert same_bits(o.field("x"), z["sorted_x"])
    counts, lists = o.neighbor_lists()
    assert np.array_equal(counts, z["nbr_counts"])
    chk = np.sum(lists.astype(np.int64) * (np.arange(len(lists)) % 7 + 1))
    assert chk == z["nbr_checksum"][()]


def test_cloud_neighbor_counts_match_brute_force_and_golden():
    """test_spatial_hash.cpp:25-51: cell-list neighbour counts and id sums equal
    brute force; here for the golden cloud, checked against the oracle too."""
    z = np.load(os.path.join(GOLDEN, "cloud.npz"))
    x = z["sorted_x"].astype(np.float32)
    ids = z["sorted_id"].astype(np.uint64)
    r2max = np.float32(z["radius"]) * np.float32(z["radius"])
    for i in range(0, len(x), 37):
        d = x[i] - x
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        m = r2 < r2max
        assert int(m.sum()) == int(z["counts"][i])
        assert int(ids[m].sum()) == int(z["id_sums"][i])


@needs_ref
@pytest.mark.parametrize("name,steps", [("c1", 3), ("box_split", 60), ("vented", 20), ("dam_break", 5),
                                        ("akinci", 10), ("options", 10), ("lh2_sphere", 5), ("ln2_boiloff", 5),
                                        ("lch4_box", 20)])
def test_oracle_bit_identical_to_reference(name, steps):
    cfg, fl, parts, lo, hi = S.SCENARIOS[name]()
    r = refpy.Ref(cfg, fl)
    r.set_threads(1)
    o = refpy.Oracle(cfg, fl)
    r.set_particles(parts, lo, hi)
    o.set_particles(parts, lo, hi)
    assert r.next_dt() == o.next_dt()
    r.step(steps)
    o.step(steps)
    n = r.num_particles()
    assert n == o.num_particles()
    for f in cabi.FIELDS:
        if f == "rmin":
            continue
        assert same_bits(r.field(f), o.field(f)), f
    dr, do = r.diagnostics().as_dict(), o.diagnostics().as_dict()
    assert dr == do


@needs_ref
def test_oracle_relax_and_maneuver_bit_identical_to_reference():
    cfg, fl, parts, lo, hi = S.c1()
    r, o = refpy.Ref(cfg, fl), refpy.Oracle(cfg, fl)
    r.set_threads(1)
    for c in (r, o):
        c.set_particles(parts, lo, hi)
        c.relax(0.01)
        c.set_maneuver([0.0, 0.01, 0.03], [[0, 0, 0], [0.05, 0, 0], [0.05, 0.01, 0]],
                       [[0, 0, 0], [0, 0, 0.02], [0, 0.01, 0.05]], origin=(0, 0, -0.01))
        c.step(6)
        c.damp_velocities(0.5)
        c.set_gravity((0.0, 0.0, -0.01))
        c.step(3)
    for f in ["x", "v", "T", "m", "p", "a", "fw", "mw"]:
        assert same_bits(r.field(f), o.field(f)), f
    assert r.diagnostics().as_dict() == o.diagnostics().as_dict()


@needs_ref
def test_fp64_reference_agrees_with_fp32_oracle():
    """Error of the FP32 path against the FP64 build of the reference (one step)."""
    cfg, fl, parts, lo, hi = S.c1()
    r64 = refpy.Ref(cfg, fl, fp64=True)
    o = refpy.Oracle(cfg, fl)
    for c in (r64, o):
        c.set_particles(parts, lo, hi)
        c.step(1)
    # align by particle id: the FP64 build may bin borderline particles differently
    a, b = np.argsort(o.field("id")), np.argsort(r64.field("id"))
    for f, tol in [("rho", 1e-5), ("sigma", 1e-5), ("x", 1e-6), ("p", 1e-3), ("T", 1e-6)]:
        assert S.normwise(o.field(f)[a], r64.field(f)[b]) < tol, f
