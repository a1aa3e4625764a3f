"""The fast field arithmetic (cryo_set_field_arithmetic(CRYO_ARITH_FAST)):
the neighbour passes compiled with FMA contraction and approximate division
and square root.  Bar: every pass output within 1e-5 (normwise, relative) of
the oracle from identical inputs, in every parity scenario; five whole steps
within the FP32 noise floor measured against the reference's FP64 build;
keys, permutation, cell tables and neighbour lists bit-exact (they do not
depend on the mode)."""
import numpy as np
import pytest

import cryo_cabi as cabi
import refpy
import scenarios as S
import test_gpu_parity as TP

pytestmark = pytest.mark.gpu

FIELD_RTOL = 1e-5


def fast_pair(name):
    cfg, fl, parts, lo, hi = S.SCENARIOS[name]()
    g = cabi.Context(cfg, fl)
    g.set_field_arithmetic(cabi.CRYO_ARITH_FAST)
    o = refpy.Oracle(cfg, fl)
    g.set_particles(parts, lo, hi)
    o.set_particles(parts, lo, hi)
    return cfg, g, o


@pytest.mark.parametrize("name", TP.SCEN)
def test_fast_pass_parity(cuda_device, name):
    cfg, g, o = fast_pair(name)
    has_vapor = bool((o.field("phase") == 1).any())
    report = []
    g.run_pass("grid_build")
    o.run_pass("grid_build")
    g.set_pass_dt(1e-4)
    o.set_pass_dt(1e-4)
    for pname, fields, where in TP.pass_plan(cfg, has_vapor):
        g.run_pass(pname)
        o.run_pass(pname)
        TP.compare(g, o, fields, where, tol=FIELD_RTOL, report=report, tag=f"fast {pname}")
        TP.resync(g, o, [f for f in fields if f not in ("phase", "flags")])
    worst = max(report, key=lambda r: r[3])
    print(f"\n[{name}, fast] worst pass output: {worst[1]} of {worst[0]} {worst[3]:.2e}")


def _by_id(ctx, f):
    return ctx.field(f)[np.argsort(ctx.field("id"), kind="stable")].astype(np.float64)


@pytest.mark.skipif(not refpy.ref_available(fp64=True), reason="FP64 reference build (oracle/_ref) not present")
@pytest.mark.parametrize("name", ["c1", "box_split", "dam_break", "lh2_sphere", "ln2_boiloff", "lch4_box"])
def test_fast_step_parity(cuda_device, name):
    """Five whole steps.  A step chains every pass, and near equilibrium the
    net acceleration is a small difference of large forces, so a field such
    as v carries the per-pass differences amplified; the FP32 oracle itself
    sits 1e-5 to 1e-4 from the reference's FP64 build after five steps (its
    single-precision noise floor, measured here on the same inputs).  Bar:
    every field within 1e-5 of the oracle or within twice that floor, and no
    further from the FP64 run than twice the floor (the fast run is as
    accurate as the exact FP32 sequence)."""
    cfg, g, o = fast_pair(name)
    cfg_, fl, parts, lo, hi = S.SCENARIOS[name]()
    r64 = refpy.Ref(cfg_, fl, fp64=True)
    r64.set_threads(16)
    r64.set_particles(parts, lo, hi)
    g.step(5)
    o.step(5)
    r64.step(5)
    assert g.num_particles() == o.num_particles()
    for f in ["phase", "id"]:
        assert np.array_equal(g.field(f), o.field(f)), f
    report = []
    for f in ["x", "v", "m", "rho", "T", "p", "sigma", "a", "ab"]:
        floor = S.normwise(_by_id(o, f), _by_id(r64, f))
        vs_oracle = S.normwise(g.field(f), o.field(f))
        vs_fp64 = S.normwise(_by_id(g, f), _by_id(r64, f))
        report.append((f, vs_oracle, vs_fp64, floor))
        assert vs_oracle <= max(FIELD_RTOL, 2.0 * floor), (name, f, vs_oracle, floor)
        assert vs_fp64 <= 2.0 * floor + 1e-6, (name, f, vs_fp64, floor)
    dg, do = g.diagnostics().as_dict(), o.diagnostics().as_dict()
    for k in ["mass_total", "enthalpy", "p_ullage", "T_sat"]:
        assert abs(dg[k] - do[k]) <= 1e-6 * max(abs(do[k]), 1e-30), (k, dg[k], do[k])
    print(f"\n[{name}, fast] 5 steps (field, vs oracle, vs FP64, oracle vs FP64):",
          [(f, f"{a:.1e}", f"{b:.1e}", f"{c:.1e}") for f, a, b, c in report])


def test_fast_dam_break_at_bench_size(cuda_device):
    """The benchmarked configuration in the fast mode: the first build's lists
    bit-exact, then 5 steps within 1e-5 of the oracle."""
    cfg, fl, parts, lo, hi = S.dam_break(dx=0.02)
    g = cabi.Context(cfg, fl)
    g.set_field_arithmetic(cabi.CRYO_ARITH_FAST)
    o = refpy.Oracle(cfg, fl)
    g.set_particles(parts, lo, hi)
    o.set_particles(parts, lo, hi)
    g.run_pass("grid_build")
    o.run_pass("grid_build")
    gc, gl = g.neighbor_lists()
    oc, ol = o.neighbor_lists()
    assert np.array_equal(gc, oc) and np.array_equal(gl, ol)
    S.assert_stored_lists(g, oc, ol, o.field("phase"))
    g2 = cabi.Context(cfg, fl)
    g2.set_field_arithmetic(cabi.CRYO_ARITH_FAST)
    o2 = refpy.Oracle(cfg, fl)
    g2.set_particles(parts, lo, hi)
    o2.set_particles(parts, lo, hi)
    g2.step(5)
    o2.step(5)
    for f in ["x", "v", "rho", "p", "a"]:
        err = S.normwise(g2.field(f), o2.field(f))
        assert err <= FIELD_RTOL, f"{f}: {err:.3e}"


def test_adjoint_refuses_the_fast_mode(cuda_device):
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    cfg.update(fixed_dt=1e-3, sound_speed=0.5, split_ratio=1e3, merge_ratio=0.0)
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    g.set_field_arithmetic(cabi.CRYO_ARITH_FAST)
    with pytest.raises(cabi.CryoError) as e:
        g.adj_forward(4, 2)
    assert e.value.code == cabi.CRYO_EINVAL
