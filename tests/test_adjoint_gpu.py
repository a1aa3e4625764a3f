"""The hand-written reverse passes of the step (csrc/cryo_adjoint.cu) against
finite differences.

Two references:
* central differences of the CUDA forward itself (FP32), Richardson-
  extrapolated from relative steps of 1e-2 and 2e-2 (rounding noise / eps and
  the eps^2 error both stay below 1e-4 of the derivative on these cases);
* central differences of the reference's own FP64 CPU build (oracle/_ref,
  step 1e-4 relative): the "reference-forward" gradient, for the parameters
  the reference can change between steps (contact angle, heater power, frame
  acceleration).

Cases are a small closed LN2 boil-off cylinder with every differentiated pass
active (density/EOS, wall extrapolation, interface normals with the
contact-angle rotation, CSF, transport velocity, momentum with artificial
viscosity and the wall guard, conduction with the heater, Lee transfer with
its normalisation, density cap and apply, the vapour mass rebalance, the
ullage model), and a "strong" variant (Lee 200 1/s both ways, subcooled
vapour, 2 kW heater) where the phase-change terms dominate.  Directions and
windows avoid the forward's kinks (upwind switches of the rebalance,
artificial-viscosity and Lee on/off thresholds), where a central difference
averages two one-sided slopes.  Tolerance: 3e-3 relative (observed values
are printed; most are below 1e-3).
"""
import ctypes as C

import numpy as np
import pytest

import cryo_cabi as cabi
import refpy
import scenarios as S

pytestmark = pytest.mark.gpu

DT = 1e-3
TOL = 3e-3
FROZEN = dict(split_ratio=1000.0, merge_ratio=0.0)  # no topology change inside a window


def weak_case():
    """The LN2 boil-off physics on a small cylinder (R 0.03 m, H 0.075 m, dx 4 mm): LN2,
    fill 0.5, 2 K superheat, Lee 5, 20 W heater, 1e-4 g, contact angle 60."""
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    cfg.update(fixed_dt=DT, sound_speed=0.5, lee_condensation=5.0, contact_angle_deg=60.0, **FROZEN)
    return cfg, fl, parts, lo, hi


def strong_case():
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1, lee_evaporation=200.0,
                         lee_condensation=200.0, heater_power=2000.0, fixed_dt=DT, sound_speed=0.5,
                         contact_angle_deg=60.0, **FROZEN)
    parts, lo, hi = S.tank([(refpy.CYLINDER, 0, 0, (0.03, 0.075, 0))], fl, 0.004,
                           refpy.make_fill(fill_fraction=0.5, T_liquid=fl.T_sat + 2, T_vapor=fl.T_sat - 2))
    return cfg, fl, parts, lo, hi


CASES = {"weak": weak_case, "strong": strong_case}


def context(case, presteps=3):
    cfg, fl, parts, lo, hi = CASES[case]()
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    g.step(presteps)
    return g


def save(g):
    size = C.c_size_t()
    g.check(g.L.cryo_state_size(g.h, C.byref(size)))
    blob = (C.c_char * size.value)()
    g.check(g.L.cryo_save_state(g.h, blob, size.value))
    return blob


def load(g, blob):
    g.check(g.L.cryo_load_state(g.h, blob, len(blob)))


def richardson(f, eps):
    """Central difference of f at 0 with steps eps and 2 eps, extrapolated."""
    d1 = (f(eps) - f(-eps)) / (2 * eps)
    d2 = (f(2 * eps) - f(-2 * eps)) / (4 * eps)
    return (4 * d1 - d2) / 3


def report(tag, ad, fd):
    rel = abs(ad - fd) / max(abs(fd), 1e-300)
    print(f"\n[{tag}] adjoint {ad:.6e} fd {fd:.6e} rel {rel:.2e}")
    return rel


def test_adjoint_rejects_unsupported_configurations(cuda_device):
    cfg, fl, parts, lo, hi = S.ln2_boiloff()
    g = cabi.Context(cfg, fl)  # adaptive dt
    g.set_particles(parts, lo, hi)
    with pytest.raises(cabi.CryoError) as e:
        g.adj_forward(2)
    assert e.value.code == cabi.CRYO_EINVAL and "fixed_dt" in str(e.value)


def test_topology_change_is_refused(cuda_device):
    """A split inside the window ends the forward with an error."""
    cfg, fl, parts, lo, hi = weak_case()
    cfg.split_ratio = 0.5  # every particle above half the reference mass splits in the first step
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    with pytest.raises(cabi.CryoError) as e:
        g.adj_forward(2, 1)
    assert "topology" in str(e.value)


def test_checkpoint_interval_does_not_change_gradients(cuda_device):
    """The reverse sweep recomputes every step bit for bit, so the gradients
    do not depend on how often the window was checkpointed, and the solver
    continues from the window's final state."""
    g = context("weak")
    blob = save(g)
    seed = np.array([1.0, -0.5, 2.0, 0.3, 0.7, -1.1, 1e-3])
    out = []
    for every in (1, 3, 20):
        load(g, blob)
        obj = g.adj_forward(7, every)
        x_end, T_end = g.field("x").copy(), g.field("T").copy()
        grads, fg = g.adj_backward(seed)
        assert np.array_equal(g.field("x"), x_end) and np.array_equal(g.field("T"), T_end)
        out.append((obj, grads, fg))
    for obj, grads, fg in out[1:]:
        assert np.array_equal(obj, out[0][0])
        assert np.array_equal(grads, out[0][1])
        assert np.array_equal(fg, out[0][2])


SCALE = {"x": 1.0, "v": 1e-2, "T": 1.0, "m": 1e3, "a": 1e-3, "ab": 1e-3}


@pytest.mark.parametrize("seed_field,dir_field", [("x", "x"), ("v", "v"), ("v", "x"), ("m", "m"), ("a", "x"),
                                                  ("a", "m"), ("ab", "x"), ("ab", "m")])
def test_one_step_state_vjp(cuda_device, seed_field, dir_field):
    """<w, s1> against a direction of s0 over one step: w on one output field
    of the end state (keyed by particle id), the direction on one input field
    of the fluid particles (relative per particle for v, m)."""
    g = context("weak")
    blob = save(g)
    n = g.num_particles()
    rng = np.random.default_rng(11)
    assert g.field("id").max() < n
    fluid0 = g.field("phase") <= 1
    shape = (n, 3) if seed_field in ("x", "v", "a", "ab") else (n,)
    w = rng.standard_normal(shape) * SCALE[seed_field]
    g.adj_forward(1, 1)
    g.adj_seed_state(seed_field, w[g.field("id")].astype(np.float32))
    g.adj_backward(np.zeros(7))
    grad = g.adj_state_gradient(dir_field).astype(np.float64)
    load(g, blob)
    base = g.field(dir_field).astype(np.float64)
    mask = fluid0.reshape((-1,) + (1,) * (base.ndim - 1))
    d = rng.standard_normal(base.shape) * mask
    if dir_field == "x":
        d *= 4e-3  # dx
    else:
        d *= np.abs(base) + 1e-3 * np.abs(base).max()

    def J(e):
        load(g, blob)
        g.set_field(dir_field, (base + e * d).astype(np.float32))
        g.adj_forward(1, 1)
        return float(np.sum(w[g.field("id")] * g.field(seed_field).astype(np.float64)))

    fd = richardson(J, 1e-2)
    ad = float(np.sum(grad * d))
    assert report(f"{seed_field} <- {dir_field}", ad, fd) <= TOL


def set_param(g, name, v, case):
    lee = 200.0 if case == "strong" else 5.0
    {"sigma": lambda: g.set_surface_tension(v), "contact_angle": lambda: g.set_contact_angle(v),
     "lee_evap": lambda: g.set_lee_coefficients(v, lee), "lee_cond": lambda: g.set_lee_coefficients(lee, v),
     "heater": lambda: g.set_heater_power(v)}[name]()


PARAM_BASE = {"sigma": 8.85e-3, "contact_angle": 60.0, "lee_evap": None, "lee_cond": None, "heater": None}
PARAM_INDEX = {"sigma": 0, "contact_angle": 1, "lee_evap": 2, "lee_cond": 3, "heater": 4}
OBJ_SEED = np.array([2e3, -1e3, 3e3, 1e4, 5e3, -2e4, 1e-3])


@pytest.mark.parametrize("case,seed_kind,name,steps", [
    ("strong", "obj", "lee_evap", 3), ("strong", "obj", "lee_cond", 10), ("strong", "obj", "heater", 10),
    ("weak", "obj", "lee_evap", 20), ("weak", "obj", "heater", 20),
    ("weak", "a", "sigma", 1), ("weak", "a", "contact_angle", 1),
    ("weak", "v", "sigma", 3), ("weak", "v", "contact_angle", 3),
])
def test_parameter_gradient(cuda_device, case, seed_kind, name, steps):
    """d(seed . objectives) or d<w, s_end> with respect to one parameter over
    a window (checkpoints every 4 steps) against central differences of the
    CUDA forward."""
    g = context(case)
    blob = save(g)
    base = PARAM_BASE[name]
    if base is None:
        base = {"lee_evap": 200.0 if case == "strong" else 5.0, "lee_cond": 200.0 if case == "strong" else 5.0,
                "heater": 2000.0 if case == "strong" else 20.0}[name]
    n = g.num_particles()
    if seed_kind == "obj":
        w, seed = None, OBJ_SEED
    else:
        w = np.random.default_rng(5).standard_normal((n, 3)) * SCALE[seed_kind]
        seed = np.zeros(7)

    def value(obj):
        if w is None:
            return float(np.dot(seed, obj))
        return float(np.sum(w[g.field("id")] * g.field(seed_kind).astype(np.float64)))

    load(g, blob)
    g.adj_forward(steps, 4)
    if w is not None:
        g.adj_seed_state(seed_kind, w[g.field("id")].astype(np.float32))
    grads, _ = g.adj_backward(seed)
    ad = grads[PARAM_INDEX[name]]

    def J(e):
        load(g, blob)
        set_param(g, name, base * (1 + e), case)
        v = value(g.adj_forward(steps, 4))
        set_param(g, name, base, case)
        return v

    fd = richardson(J, 1e-2) / base
    assert report(f"{case} {seed_kind} d/d{name} {steps} steps", ad, fd) <= TOL


# ------------------------------------------------ reference-forward FD
def reference_run(cfg, fl, parts, lo, hi, steps, after_init=None, w=None):
    """The reference's FP64 CPU build over `steps` steps from a freshly
    initialised state (`after_init` applied once initialised): returns
    seed . [int F, int M, p_ullage] and, with w, <w, v_end> keyed by id."""
    r = refpy.Ref(cfg, fl, fp64=True)
    r.set_particles(parts, lo, hi)
    r.next_dt()
    if after_init:
        after_init(r)
    F = np.zeros(3)
    M = np.zeros(3)
    for _ in range(steps):
        r.step(1)
        d = r.diagnostics()
        F += DT * np.asarray(d.slosh_force, np.float64)
        M += DT * np.asarray(d.slosh_moment, np.float64)
    p = r.diagnostics().p_ullage
    obj = float(np.dot(OBJ_SEED, np.concatenate([F, M, [p]])))
    vdot = float(np.sum(w[r.field("id")] * r.field("v"))) if w is not None else 0.0
    r.close()
    return obj, vdot


REF_CASES = [
    # (case, parameter, steps, seed): parameters the reference changes after its initialisation
    ("weak", "contact_angle", 10, "obj"), ("weak", "heater", 10, "obj"), ("weak", "frame_x", 10, "obj"),
    ("weak", "frame_y", 3, "v"), ("weak", "frame_z", 3, "v"),
    # ... and those it fixes at construction (not read by the initialisation, or corrected for it)
    ("weak", "lee_evap", 10, "obj"), ("strong", "lee_evap", 5, "obj"), ("strong", "lee_cond", 5, "obj"),
    ("weak", "sigma", 10, "obj"), ("weak", "sigma", 3, "v"),
]


@pytest.mark.skipif(not refpy.ref_available(fp64=True), reason="reference FP64 build absent")
@pytest.mark.parametrize("case,name,steps,seed_kind", REF_CASES)
def test_gradient_matches_reference_fp64_finite_difference(cuda_device, case, name, steps, seed_kind):
    """The adjoint of this library's FP32 steps against central differences
    (relative step 1e-4) of the reference's own double-precision forward,
    both from the same freshly initialised state.  The surface tension is a
    constructor argument of the reference, so its initial rate evaluation
    (the CSF part of the first step's kick) moves with it; that term is added
    to the window's gradient from the initial-state adjoint."""
    cfg, fl, parts, lo, hi = CASES[case]()
    g = cabi.Context(cfg, fl)
    g.set_particles(parts, lo, hi)
    g.next_dt()  # initialise
    nrm0, kappa0 = g.field("nrm").astype(np.float64), g.field("kappa").astype(np.float64)
    n = g.num_particles()
    w = np.random.default_rng(9).standard_normal((n, 3)) * 1e-2 if seed_kind == "v" else None
    seed = OBJ_SEED if seed_kind == "obj" else np.zeros(7)
    g.adj_forward(steps, 4)
    if w is not None:
        g.adj_seed_state("v", w[g.field("id")].astype(np.float32))
    grads, fg = g.adj_backward(seed)
    lee = (cfg.lee_evaporation, cfg.lee_condensation)
    if name.startswith("frame_"):
        c = "xyz".index(name[-1])
        ad, base, eps = fg.sum(axis=0)[c], 0.0, 1e-6

        def run(v):
            a = [0.0, 0.0, 0.0]
            a[c] = v
            return reference_run(cfg, fl, parts, lo, hi, steps, lambda r: r.set_frame_motion(a=tuple(a)), w)
    elif name in ("contact_angle", "heater"):
        ad, base = (grads[1], 60.0) if name == "contact_angle" else (grads[4], cfg.heater_power)
        eps = 1e-4 * base
        setter = "set_contact_angle" if name == "contact_angle" else "set_heater_power"
        run = lambda v: reference_run(cfg, fl, parts, lo, hi, steps, lambda r: getattr(r, setter)(v), w)
    else:
        if name == "sigma":
            abar0 = g.adj_state_gradient("a").astype(np.float64)
            csf_unit = 2.0 / (fl.rho_liquid + fl.rho_vapor)
            ad = grads[0] + float(np.sum(np.einsum("ij,ij->i", abar0, nrm0) * kappa0)) * csf_unit
            base = fl.sigma
        else:
            ad = grads[2] if name == "lee_evap" else grads[3]
            base = lee[0] if name == "lee_evap" else lee[1]
        eps = 1e-4 * base

        def run(v):
            c2, f2 = cabi.Config(), cabi.Fluid()
            C.pointer(c2)[0], C.pointer(f2)[0] = cfg, fl
            if name == "sigma":
                f2.sigma = v
            elif name == "lee_evap":
                c2.lee_evaporation = v
            else:
                c2.lee_condensation = v
            return reference_run(c2, f2, parts, lo, hi, steps, None, w)
    k = 0 if seed_kind == "obj" else 1
    fd = (run(base + eps)[k] - run(base - eps)[k]) / (2 * eps)
    assert report(f"reference FP64 {case} d({seed_kind})/d{name} {steps} steps", ad, fd) <= 1e-3
