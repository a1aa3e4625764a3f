"""The torch.autograd.Function over the adjoint (cryo_adjoint.SloshWindow)
through the reference's Python API (CryoSPH.Solver): its gradients are the
Solver's adjoint results mapped to the parameters (sigma, contact angle, one
Lee coefficient for both directions, piecewise-constant frame-acceleration
knots), and a knot gradient matches central differences of the reference's
own FP64 forward driven by the same ManeuverProfile."""
import numpy as np
import pytest
import torch

import CryoSPH as cs
import cryo_adjoint as ca
import cryo_cabi as cabi
import refpy
import scenarios as S

pytestmark = pytest.mark.gpu

DT = 1e-3
STEPS, KNOTS, EVERY = 8, 4, 3
SEED = np.array([2e3, -1e3, 3e3, 1e4, 5e3, -2e4, 1e-3])


def particles():
    return S.ln2_boiloff()[2:]


def solver():
    fluid = cs.FluidProperties.liquid_nitrogen()
    cfg = cs.SolverConfig()
    cfg.dx = 0.004
    cfg.gravity = (0.0, 0.0, -9.81e-4)
    cfg.thermo_mode = cs.TankThermoMode.Closed
    cfg.heater_power = 20.0
    cfg.lee_evaporation = 5.0
    cfg.lee_condensation = 5.0
    cfg.contact_angle_deg = 60.0
    cfg.fixed_dt = DT
    cfg.sound_speed = 0.5
    cfg.split_ratio = 1e3
    cfg.merge_ratio = 0.0
    s = cs.Solver(cfg, fluid)
    p, lo, hi = particles()
    s.set_particles(p["x"].astype(np.float64), p["m"].astype(np.float64), p["rho"].astype(np.float64),
                    p["T"].astype(np.float64), p["phase"], domain_lo=lo, domain_hi=hi, normal=p["nrm"].astype(np.float64),
                    flags=p["flags"])
    s.next_dt()  # initialise
    return s, fluid


def test_function_gradients_are_the_solver_adjoint(cuda_device):
    s, fluid = solver()
    blob = s.save_state()
    kn = np.zeros((KNOTS, 3))
    kn[:, 0] = [0.01, -0.02, 0.015, 0.0]
    sigma = torch.tensor(float(fluid.sigma), dtype=torch.float64, requires_grad=True)
    theta = torch.tensor(60.0, dtype=torch.float64, requires_grad=True)
    lee = torch.tensor(5.0, dtype=torch.float64, requires_grad=True)
    kt = torch.tensor(kn, requires_grad=True)
    s.load_state(blob)
    out = ca.slosh_window(s, sigma, theta, lee, kt, STEPS, EVERY)
    (out * torch.tensor(SEED)).sum().backward()
    # the same window through the Solver directly
    s.load_state(blob)
    times, seg = ca.knot_schedule(s.time, float(s.config.fixed_dt), STEPS, KNOTS)
    s.set_maneuver(ca._maneuver(times, kn))
    obj = s.adjoint_forward(STEPS, EVERY)
    assert np.array_equal(obj, out.detach().numpy())
    g = s.adjoint_backward(list(SEED))
    assert float(sigma.grad) == g["sigma"]
    assert float(theta.grad) == g["contact_angle"]
    assert float(lee.grad) == g["lee_evaporation"] + g["lee_condensation"]
    expect = np.zeros((KNOTS, 3))
    np.add.at(expect, seg, g["frame_acceleration"])
    assert np.array_equal(kt.grad.numpy(), expect)
    print("\n[torch] grads:", float(sigma.grad), float(theta.grad), float(lee.grad), kt.grad[:, 0].tolist())


@pytest.mark.skipif(not refpy.ref_available(fp64=True), reason="reference FP64 build absent")
def test_knot_gradient_matches_reference_fp64_finite_difference(cuda_device):
    s, fluid = solver()
    kn = np.zeros((KNOTS, 3))
    kn[:, 0] = [0.01, -0.02, 0.015, 0.0]
    t0 = s.time
    kt = torch.tensor(kn, requires_grad=True)
    out = ca.slosh_window(s, fluid.sigma, 60.0, 5.0, kt, STEPS, EVERY)
    (out * torch.tensor(SEED)).sum().backward()
    times, _ = ca.knot_schedule(t0, float(s.config.fixed_dt), STEPS, KNOTS)
    cfg = cabi.py_config(dx=0.004, gravity=(0, 0, -9.81e-4), thermo_mode=1, heater_power=20.0, lee_evaporation=5.0,
                         lee_condensation=5.0, contact_angle_deg=60.0, fixed_dt=DT, sound_speed=0.5,
                         split_ratio=1e3, merge_ratio=0.0)
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    p, lo, hi = particles()

    def J(k, c, e):
        k2 = kn.copy()
        k2[k, c] += e
        r = refpy.Ref(cfg, fl, fp64=True)
        r.set_particles(p, lo, hi)
        r.next_dt()
        r.set_maneuver(times, np.repeat(k2, 2, axis=0))
        F, M = np.zeros(3), np.zeros(3)
        for _ in range(STEPS):
            r.step(1)
            d = r.diagnostics()
            F += DT * np.asarray(d.slosh_force, np.float64)
            M += DT * np.asarray(d.slosh_moment, np.float64)
        val = float(np.dot(SEED, np.concatenate([F, M, [r.diagnostics().p_ullage]])))
        r.close()
        return val

    for k, c in ((1, 0), (2, 1)):
        eps = 1e-6
        fd = (J(k, c, eps) - J(k, c, -eps)) / (2 * eps)
        ad = float(kt.grad[k, c])
        rel = abs(ad - fd) / abs(fd)
        print(f"\n[knot {k}, {c}] adjoint {ad:.6e} reference fp64 fd {fd:.6e} rel {rel:.2e}")
        assert rel <= 1e-3
