"""Throughput of the per-step particle update on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload dam_break|c1|c3] [--impl ours|reference]

Workload (default): the SPHERIC Test 2 dam break with an obstacle at dx 0.02 m
(203 662 particles with walls, 82 350 fluid), continuity density, free-slip
walls, no surface tension or heat, fluid lattice jittered +-0.05 dx from
numpy PCG64(2002).  One step = one Solver::step.  The metric counts wall
particles (as the reference's perf_scaling.cpp does).

Timing: W untimed steps, then K steps, each bracketed by CUDA events on the
solver's stream, with a 256 MiB memset between steps (outside the events) so
every step starts with a cold L2 -- the dam-break state (~61 MB) would
otherwise stay resident in the 126 MB L2.  value = particles * K / sum(step
times).  Multi-GPU (torchrun): every rank runs its own replica, barrier on both
sides, max over ranks.

Also reported: e2e (the same steps through the public API with host buffers:
per step the frame-motion input goes host->device and the diagnostics come
back device->host, plus the initial state upload and the final download),
the roofline of the dominant kernel (per-kernel CUDA-event times from a
profiled run, algorithmic bytes from cryo_roofline.py, DRAM traffic from the
committed ncu summary), SM clocks sampled during the timed region, the
reference's own CPU implementation timed on this host (rank 0, N=1), and
`batched`: the 64-tank ensemble (seeded tanks of 5k-200k particles) advanced
by one cs.Ensemble -- one graph launch per ensemble step, branch count
autotuned -- against the same tanks stepped back to back by plain Solvers,
with every tank's diagnostics compared bit for bit.  Under torchrun the
tanks are sharded over ranks (longest-processing-time first); the step has
no collective.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "microgravity-cryogenic-multi-phase-sph-solver_b200")
sys.path.insert(0, PKG)

METRIC = "particle-steps/s/GPU (plain)"
UNIT = "particle-steps/s"
SEED = 2002


# ----------------------------------------------------------------- workloads
# Each workload is plain data: the C ABI's config fields, a fluid preset with
# overrides, the tank as a geometry node list (kind, a, b, p) whose last node
# is the root (kinds as CRYO_GEOM_*: a/b index child nodes), the fill, a
# particle filter and the domain.  Both arms build from it: this library's arm
# through its CryoSPH module, the reference arm through the reference's own
# lattice generator in oracle/_ref and nothing of this package.  The fluid
# lattice is then jittered +-0.05 dx by numpy PCG64(SEED) (walls stay on it).
G_CYLINDER, G_CAPSULE, G_SPHERE, G_BOX, G_TRANSLATED, G_DIFFERENCE, G_UNION = range(7)
FLUID_LH2, FLUID_LN2, FLUID_H2O = 1, 2, 5
FILL_FULL = 2


def workload_spec(name, dx=None):
    if name == "dam_break":
        # SPHERIC Test 2 (validation/spheric_test2/run.py:36-73 of the reference)
        dx = dx or 0.02
        x_front, box = 0.744, (0.161, 0.403, 0.161)
        pad = 4 * dx
        return dict(
            label=f"dam_break_spheric2_dx{dx:g}", fluid=(FLUID_H2O, {"mu_liquid": 1.0e-3}),
            config=dict(dx=dx, gravity=(0.0, 0.0, -9.81), surface_tension=0, thermal=0, phase_change=0,
                        density_mode=1, velocity_scale=(2 * 9.81 * 0.55) ** 0.5, artificial_viscosity=0.02,
                        delta_sph=0.1, no_slip=0),
            nodes=[(G_BOX, 0, 0, (3.22, 1.0, 1.0)), (G_TRANSLATED, 0, 0, (1.61, 0.0, 0.5)),
                   (G_BOX, 0, 0, box), (G_TRANSLATED, 2, 0, (x_front - box[0] / 2, 0.0, box[2] / 2)),
                   (G_DIFFERENCE, 1, 3, (0.0, 0.0, 0.0))],
            fill=dict(mode=FILL_FULL), keep=_dam_break_column,
            domain=((-pad, -0.5 - pad, -pad), (3.22 + pad, 0.5 + pad, 1.0 + pad)))
    if name == "c1":
        dx = dx or 0.004
        return dict(label=f"c1_ln2_cylinder_dx{dx:g}", fluid=(FLUID_LN2, {}),
                    config=dict(dx=dx, gravity=(0.0, 0.0, -9.81e-4), heater_power=20.0, thermo_mode=1),
                    nodes=[(G_CYLINDER, 0, 0, (0.05, 0.12, 0.0))], fill=dict(fill_fraction=0.5), keep=None,
                    domain=None)
    if name == "c3":
        dx = dx or 0.0052
        return dict(label=f"c3_lh2_sphere_dx{dx:g}", fluid=(FLUID_LH2, {}),
                    config=dict(dx=dx, gravity=(0.0, 0.0, -9.81e-4), heater_power=0.0, thermo_mode=1),
                    nodes=[(G_SPHERE, 0, 0, (0.5, 0.0, 0.0))], fill=dict(fill_fraction=0.5), keep=None,
                    domain=None)
    raise SystemExit(f"unknown workload {name}")


def _dam_break_column(x, phase):
    """Walls, and the water column 1.228 m long and 0.55 m high at the far end."""
    return (phase == 2) | ((x[:, 0] > 3.22 - 1.228) & (x[:, 2] < 0.55))


def _jitter(x, phase, dx):
    rng = np.random.Generator(np.random.PCG64(SEED))
    fl = phase != 2
    x = np.asarray(x, np.float32).copy()
    x[fl] += rng.uniform(-0.05 * dx, 0.05 * dx, size=(int(fl.sum()), 3)).astype(np.float32)
    return x


def _cs_geometry(cs, nodes):
    objs = []
    for kind, a, b, p in nodes:
        if kind == G_CYLINDER:
            objs.append(cs.CylinderTank(p[0], p[1]))
        elif kind == G_CAPSULE:
            objs.append(cs.CapsuleTank(p[0], p[1]))
        elif kind == G_SPHERE:
            objs.append(cs.SphereTank(p[0]))
        elif kind == G_BOX:
            objs.append(cs.BoxTank(*p))
        elif kind == G_TRANSLATED:
            objs.append(cs.Translated(objs[a], tuple(p)))
        elif kind == G_DIFFERENCE:
            objs.append(cs.Difference(objs[a], objs[b]))
        else:
            objs.append(cs.Union(objs[a], objs[b]))
    return objs[-1]


def workload(name, cs, dx_override=None):
    """This library's arm: (label, SolverConfig, fluid, particle dict, domain lo, hi)."""
    w = workload_spec(name, dx_override)
    which, over = w["fluid"]
    fluid = {FLUID_LH2: cs.FluidProperties.liquid_hydrogen, FLUID_LN2: cs.FluidProperties.liquid_nitrogen,
             FLUID_H2O: cs.FluidProperties.water}[which]()
    for k, v in over.items():
        setattr(fluid, k, v)
    cfg = cs.SolverConfig()
    for k, v in w["config"].items():
        cur = getattr(cfg, k)
        setattr(cfg, k, tuple(v) if k == "gravity" else (type(cur)(int(v)) if hasattr(cur, "value") else
                                                          (bool(v) if isinstance(cur, bool) else v)))
    geo = _cs_geometry(cs, w["nodes"])
    fill = cs.FillSpec()
    for k, v in w["fill"].items():
        setattr(fill, k, [cs.FillMode.Settled, cs.FillMode.CentralBubble, cs.FillMode.Full][v] if k == "mode" else v)
    dx = w["config"]["dx"]
    p = cs.tank_particles(geo, fluid, dx, fill)
    if w["keep"] is not None:
        keep = w["keep"](p["position"], p["phase"])
        p = {k: v[keep] for k, v in p.items()}
    lo, hi = w["domain"] if w["domain"] else cs.tank_domain(geo, dx, 3)
    p["position"] = _jitter(p["position"], p["phase"], dx)
    return w["label"], cfg, fluid, p, lo, hi


def ref_workload(name, dx_override=None):
    """The reference arm's inputs from the same spec, through the reference's
    own generator (build_tank_particles, geometry.cpp:242-330, in oracle/_ref):
    (label, refpy config, refpy fluid, particle arrays, lo, hi)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_abi
    import refpy
    w = workload_spec(name, dx_override)
    which, over = w["fluid"]
    fluid = ref_abi.fluid(which, **over)
    cfg = ref_abi.config(**w["config"])
    dx = w["config"]["dx"]
    fkw = dict(w["fill"])
    parts = refpy.tank_particles(w["nodes"], fluid, dx, refpy.make_fill(**fkw))
    if w["keep"] is not None:
        keep = w["keep"](parts["x"], parts["phase"])
        parts = {k: v[keep] for k, v in parts.items()}
    lo, hi = w["domain"] if w["domain"] else refpy.tank_domain(w["nodes"], dx, 3)
    parts["x"] = _jitter(parts["x"], parts["phase"], dx)
    return w["label"], cfg, fluid, parts, lo, hi


def config_block(label, n_total, n_fluid, n_wall, world):
    """The `config` of the JSON line; both arms print the same dict."""
    return {"workload": label, "particles": n_total, "fluid": n_fluid, "walls": n_wall,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "seed": SEED}


def c4_tanks(cs, count=64, n_lo=5_000, n_hi=200_000, seed=SEED):
    """The 64-tank ensemble as seeded synthetic tanks: shape cylinder or sphere,
    radius U[0.03, 0.3] m (cylinder height 2R x U[1, 2.5]), fill U[0.2, 0.8],
    dx chosen so the particle count (walls included) is log-uniform in
    [n_lo, n_hi], fluid LN2 / LOX / LCH4, gravity 1e-4 g, a lateral pulse of
    U[0, 0.1] m/s^2 (ramped in over 10 ms, held to 50 ms, out by 60 ms)."""
    rng = np.random.Generator(np.random.PCG64(seed + 4))
    presets = [cs.FluidProperties.liquid_nitrogen, cs.FluidProperties.liquid_oxygen,
               cs.FluidProperties.liquid_methane]
    tanks = []
    for t in range(count):
        sphere = bool(rng.random() < 0.5)
        R = float(rng.uniform(0.03, 0.3))
        H = float(2.0 * R * rng.uniform(1.0, 2.5))
        fill_fraction = float(rng.uniform(0.2, 0.8))
        n_target = math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))
        which = int(rng.integers(3))
        amp = float(rng.uniform(0.0, 0.1))
        if sphere:
            geo, vol, area = cs.SphereTank(R), 4.0 / 3.0 * math.pi * R ** 3, 4.0 * math.pi * R ** 2
        else:
            geo, vol, area = cs.CylinderTank(R, H), math.pi * R * R * H, 2.0 * math.pi * R * (H + R)
        lo_dx, hi_dx = 1e-5, 1.0  # interior lattice + 3 wall layers ~ n_target
        for _ in range(60):
            dx = math.sqrt(lo_dx * hi_dx)
            if vol / dx ** 3 + 3.0 * area / dx ** 2 > n_target:
                lo_dx = dx
            else:
                hi_dx = dx
        dx = math.sqrt(lo_dx * hi_dx)
        fluid = presets[which]()
        cfg = cs.SolverConfig()
        cfg.dx = dx
        cfg.gravity = (0.0, 0.0, -9.81e-4)
        cfg.thermo_mode = cs.TankThermoMode.Closed
        fill = cs.FillSpec()
        fill.fill_fraction = fill_fraction
        p = cs.tank_particles(geo, fluid, dx, fill)
        lo, hi = cs.tank_domain(geo, dx, 3)
        jr = np.random.Generator(np.random.PCG64(seed + 1000 + t))
        fl = p["phase"] != 2
        x = p["position"].astype(np.float32).copy()
        x[fl] += jr.uniform(-0.05 * dx, 0.05 * dx, size=(int(fl.sum()), 3)).astype(np.float32)
        p["position"] = x
        man = cs.ManeuverProfile([0.0, 0.01, 0.05, 0.06],
                                 np.array([[0, 0, 0], [amp, 0, 0], [amp, 0, 0], [0, 0, 0]], np.float64))
        tanks.append(dict(cfg=cfg, fluid=fluid, p=p, lo=lo, hi=hi, maneuver=man, n=int(len(x)),
                          shape="sphere" if sphere else "cylinder", fluid_name=["LN2", "LOX", "LCH4"][which]))
    return tanks


def load(solver, p, lo, hi):
    solver.set_particles(p["position"], p["mass"], p["density"], p["temperature"], p["phase"], domain_lo=lo,
                         domain_hi=hi, normal=p["normal"], flags=p["flags"])


# ---------------------------------------------------------------- clocks
class Clocks:
    """SM clock and clock-event reasons sampled while the timed steps run.
    NVML is read every ~1 ms from a background thread (the timed region of a
    short run lasts a few milliseconds); where NVML cannot be opened,
    nvidia-smi samples every 200 ms."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None
        self.nvml = None
        self.rows = []

    def _open_nvml(self):
        import threading
        import pynvml
        import torch
        pynvml.nvmlInit()
        prop = torch.cuda.get_device_properties(self.device)
        bus = f"{prop.pci_domain_id:08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
        h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        self.bits = {name: getattr(pynvml, attr) for name, attr in self.REASONS}

        def sample():
            self.rows.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                              int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))))

        sample()
        self.stop = threading.Event()

        def run():
            while not self.stop.is_set():
                sample()
                time.sleep(0.001)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        self.nvml = pynvml

    def __enter__(self):
        try:
            self._open_nvml()
            return self
        except Exception:
            self.nvml = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.nvml:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.nvml:
            rows = list(self.rows)
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
            reasons = sorted({name for _, r in rows for name, bit in self.bits.items() if r & bit})
            return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(rows), "source": "NVML, every ~1 ms"}
        rows = []
        try:
            with open(self.path) as fh:
                for line in fh:
                    parts = [s.strip() for s in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except (OSError, TypeError):
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, every 200 ms"}


# ------------------------------------------------------------- reference arm
def reference_rate(name, dx, steps, warmup, budget_s=60.0, cuda=False, inputs=None):
    """The reference's own implementation (oracle/_ref, built from its own
    sources) on the workload built by ref_workload(): its CPU/OpenMP backend
    with every host thread, or (cuda=True) its CUDA backend built for
    sm_100a, wall clock as its perf_scaling.cpp times it.  At most `steps`
    steps, fewer when one step times `budget_s` would be exceeded.  Returns
    (rate, threads, steps timed, seconds, label, particle counts) or None."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refpy
    if not refpy.ref_available(cuda=cuda):
        return None
    label, cfg, fluid, parts, lo, hi = inputs or ref_workload(name, dx)
    ref = refpy.Ref(cfg, fluid, cuda=cuda)
    threads = os.cpu_count() or 1
    ref.set_threads(threads)
    ref.set_particles(parts, lo, hi)
    ref.step(max(1, min(warmup, 2)))
    t0 = time.perf_counter()
    ref.step(1)
    one = time.perf_counter() - t0
    k = int(max(2, min(steps, budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    ref.step(k)
    el = time.perf_counter() - t0
    n = ref.num_particles()
    n_wall = int((parts["phase"] == 2).sum())
    return n * k / el, threads, k, el, label, (len(parts["x"]), len(parts["x"]) - n_wall, n_wall)


def reference_main(args, world):
    """--impl reference: the reference's CPU implementation of the path on this
    host's cores, on the same workload and config as this library's arm.
    Nothing of this package is imported or loaded in this process."""
    if args.workload == "c4":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched ensemble (one Solver "
                                                              "per tank); its back-to-back solves are this "
                                                              "library's own back_to_back leg"}))
        return 0
    r = reference_rate(args.workload, args.dx, args.steps, args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) not present"}))
        return 0
    rate, threads, k, el, label, (n_total, n_fluid, n_wall) = r
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": k,
        "warmup": args.warmup, "ms_per_step": el / k * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 fields, f64 reductions", "data": "synthetic",
        "config": config_block(label, n_total, n_fluid, n_wall, world),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{k} steps of {label} after 2 warm-up steps (its OpenMP backend, "
                                   f"{threads} threads)"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timing": "wall clock around the steps; inputs from the reference's own lattice generator",
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--workload", default="dam_break", choices=["dam_break", "c1", "c3", "c4"],
                    help="c4: only the batched-ensemble comparison (64 tanks), reported as the main line")
    ap.add_argument("--dx", type=float, default=None, help="lattice spacing override (dam_break, c1, c3)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arith", default="fast", choices=["fast", "exact"],
                    help="field arithmetic of the neighbour passes for the timed steps and e2e: fast (contracted, "
                         "within 1e-5 of the reference) or exact (the reference's IEEE sequence, bit-identical)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=50)
    ap.add_argument("--batched-steps", type=int, default=100,
                    help="steps of the batched-ensemble comparison (0 = skip it)")
    ap.add_argument("--batched-tanks", type=int, default=64)
    ap.add_argument("--adjoint-steps", type=int, default=400,
                    help="steps of the differentiated LN2 boil-off window (0 = skip the adjoint leg)")
    ap.add_argument("--adjoint-every", type=int, default=20, help="checkpoint interval of the adjoint window")
    ap.add_argument("--adjoint-fd64", type=int, default=0,
                    help="run only the FP64 finite-difference check of the adjoint over a window of this many steps "
                         "from the boil-off tank's initial lattice, and print its record")
    ap.add_argument("--only-adjoint", action="store_true",
                    help="run only the adjoint leg (LN2 boil-off window) and print its record; for profiler launch lists")
    ap.add_argument("--slabs", type=int, default=0,
                    help="also step the workload as one tank cut into this many slabs (0 = skip)")
    ap.add_argument("--slab-devices", default=None,
                    help="comma-separated device per slab (default: every slab on this rank's device)")
    ap.add_argument("--slab-steps", type=int, default=50, help="timed steps of the slab leg")
    ap.add_argument("--side-force-steps", type=int, default=0,
                    help="with --workload c3: steps of the manoeuvre run (side force against -M a; 0 = skip)")
    ap.add_argument("--probe-steps", type=int, default=1500,
                    help="steps of the dam break's probe-pressure series against the FP64 reference (0 = skip)")
    ap.add_argument("--probe-dx", type=float, default=0.04, help="lattice spacing of the probe-series dam break")
    ap.add_argument("--only-timed", action="store_true",
                    help="run the timed steps only (no e2e, roofline or CPU legs); for profiler launch lists")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # rank 0 alone times the reference; nothing of this package is loaded
        return reference_main(args, world) if rank == 0 else 0

    import CryoSPH as cs

    if args.adjoint_fd64 > 0:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"adjoint_fd64": adjoint_fd64_run(cs, local, args.adjoint_fd64, args.adjoint_every)}))
        return 0
    if args.only_adjoint:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"adjoint": adjoint_run(cs, local, args.adjoint_steps, args.adjoint_every)}))
        return 0
    if args.workload == "c4":
        return batched_main(args, cs, rank, world, local)
    label, cfg, fluid, p, lo, hi = workload(args.workload, cs, args.dx)
    n_total = int(len(p["position"]))
    n_wall = int((p["phase"] == 2).sum())
    n_fluid = n_total - n_wall
    has_vapor = bool((p["phase"] == 1).any())

    import torch
    import cryo_cabi as cabi

    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    device = local

    L = cabi.load()
    arith = cs.FieldArithmetic.Fast if args.arith == "fast" else cs.FieldArithmetic.Exact
    solver = cs.Solver(cfg, fluid, device)
    solver.field_arithmetic = arith
    load(solver, p, lo, hi)
    stream = torch.cuda.ExternalStream(solver.stream_handle, device=device)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)

    solver.run_steps(args.warmup)
    torch.cuda.synchronize()

    # ---- timed: device time of K steps, L2 flushed between steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(device) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                solver.step()
                ends[k].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    clocks = clk.summary()
    n_now = solver.num_particles
    t = torch.tensor([total_ms], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * n_total * args.steps / (max_ms / 1e3)
    per_step = ctypes_int(L, "cryo_kernels_per_step", solver.handle)

    e2e = roof = other = None
    if rank == 0 and not args.only_timed:
        # ---- e2e through the public API with host buffers
        e2e = e2e_run(cs, cfg, fluid, p, lo, hi, args.steps, device, stream, flush, args.warmup, arith)
        # ---- roofline of the dominant kernel (profiled run, CUDA events per kernel)
        roof = roofline(cs, cabi, L, cfg, fluid, p, lo, hi, args.profile_steps, n_fluid, n_wall, has_vapor, label,
                        arith)
        # ---- the same timed steps in the other field arithmetic
        other_arith = cs.FieldArithmetic.Exact if args.arith == "fast" else cs.FieldArithmetic.Fast
        solver.field_arithmetic = other_arith
        solver.run_steps(args.warmup)
        torch.cuda.synchronize()
        ms_o = 0.0
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                solver.step()
                ends[k].record(stream)
        torch.cuda.synchronize()
        ms_o = sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends))
        other = {"field_arithmetic": "exact" if args.arith == "fast" else "fast",
                 "value": n_total * args.steps / (ms_o / 1e3), "ms_per_step": ms_o / args.steps}

    # ---- batched ensemble (64 tanks): tanks sharded over ranks, no collective in the step
    batched = None
    if args.batched_steps > 0 and not args.only_timed:
        import cryo_shard
        del solver
        torch.cuda.empty_cache()
        all_tanks = c4_tanks(cs, count=args.batched_tanks)
        mine = cryo_shard.shard_of([tk["n"] for tk in all_tanks], rank, world)
        b = batched_run(cs, [all_tanks[t] for t in mine], args.batched_steps, args.warmup, device, arith=arith)
        agg = torch.tensor([b["ms_per_step"], b["back_to_back_ms_per_step"], 0.0 if b["diagnostics_bit_identical"] else 1.0],
                           dtype=torch.float64, device=device)
        if dist:
            dist.all_reduce(agg, op=dist.ReduceOp.MAX)
        ms_e, ms_s, differs = (float(v) for v in agg.tolist())
        n_all = sum(tk["n"] for tk in all_tanks)
        batched = dict(b)
        batched.update({
            "tanks": len(all_tanks), "particles": n_all, "ranks": world,
            "particles_min": min(tk["n"] for tk in all_tanks), "particles_max": max(tk["n"] for tk in all_tanks),
            "value": n_all / (ms_e / 1e3), "ms_per_step": ms_e,
            "back_to_back": n_all / (ms_s / 1e3), "back_to_back_ms_per_step": ms_s, "speedup": ms_s / ms_e,
            "diagnostics_bit_identical": differs == 0.0,
            "sharding": "tanks split over ranks longest-processing-time first by particle count" if world > 1 else None,
        })

    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.only_timed:
        r = reference_rate(args.workload, args.dx, 2000, 3, budget_s=10.0, cuda=True)
        if r is not None:
            rate, _, k, el = r[:4]
            ref_gpu = {"value": rate, "unit": UNIT, "kind": "reference CUDA backend (its own sources, sm_100a)",
                       "sample": f"{k} steps of {label} after 3 warm-up steps ({el:.1f} s wall clock)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.only_timed:
        r = reference_rate(args.workload, args.dx, 200, 2, budget_s=20.0)
        if r is not None:
            rate, threads, k, el = r[:4]
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{k} steps of {label} after 2 warm-up steps ({el:.1f} s, OpenMP)"}

    # one tank over several slabs (halo layers exchanged between passes)
    slabs = None
    if rank == 0 and args.slabs > 0 and not args.only_timed:
        devs = [int(d) for d in args.slab_devices.split(",")] if args.slab_devices else [device] * args.slabs
        slabs = slab_run(cs, cfg, fluid, p, lo, hi, args.slabs, devs, args.slab_steps, label)

    side = None
    if rank == 0 and args.workload == "c3" and args.side_force_steps > 0:
        side = side_force_run(cs, device, args.side_force_steps, arith, args.dx)

    # the dam break's probe-pressure series against the reference's FP64 build
    probes = None
    if rank == 0 and world == 1 and args.probe_steps > 0 and not args.only_timed and args.workload == "dam_break":
        probes = probe_series_run(cs, device, args.probe_dx, args.probe_steps, arith)

    # the adjoint leg last: its window holds several GB until it is released
    adjoint = None
    if rank == 0 and args.adjoint_steps > 0 and not args.only_timed:
        torch.cuda.empty_cache()
        adjoint = adjoint_run(cs, device, args.adjoint_steps, args.adjoint_every)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 fields, f64 reductions", "data": "synthetic",
            "config": config_block(label, n_total, n_fluid, n_wall, world),
            "particles_after": int(n_now),
            "field_arithmetic": args.arith,
            "other_arithmetic": other,
            "timing": {"l2": "flushed between timed steps (256 MiB memset outside the events)",
                       "execution": "CUDA graph per step"},
            "per_gpu": value / world,
            "gpu_launches": per_step * args.steps,
            "clocks": {k: clocks.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons", "samples", "source")},
            "e2e": e2e,
            "roofline": roof,
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "batched": batched,
            "adjoint": adjoint,
            "slabs": slabs,
            "probe_series": probes,
            "side_force": side,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batched_main(args, cs, rank, world, local):
    """--workload c4: the batched ensemble against back-to-back plain solves
    as the main line (metric: batched particle-steps/s)."""
    import torch
    import cryo_shard
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    all_tanks = c4_tanks(cs, count=args.batched_tanks)
    mine = cryo_shard.shard_of([tk["n"] for tk in all_tanks], rank, world)
    if dist:
        dist.barrier()
    with Clocks(local) as clk:
        arith = cs.FieldArithmetic.Fast if args.arith == "fast" else cs.FieldArithmetic.Exact
        b = batched_run(cs, [all_tanks[t] for t in mine], args.steps, args.warmup, local, arith=arith)
    agg = torch.tensor([b["ms_per_step"], b["back_to_back_ms_per_step"], 0.0 if b["diagnostics_bit_identical"] else 1.0],
                       dtype=torch.float64, device=local)
    if dist:
        dist.all_reduce(agg, op=dist.ReduceOp.MAX)
    ms_e, ms_s, differs = (float(v) for v in agg.tolist())
    n_all = sum(tk["n"] for tk in all_tanks)
    if rank == 0:
        clocks = clk.summary()
        print(json.dumps({
            "metric": "particle-steps/s/GPU (batched)", "value": n_all / (ms_e / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": b["steps"], "warmup": args.warmup, "ms_per_step": ms_e, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 reductions", "data": "synthetic",
            "config": {"workload": b["workload"], "tanks": len(all_tanks), "particles": n_all,
                       "parallelism": f"tanks sharded x{world}" if world > 1 else "1 GPU",
                       "l2": "state of all tanks (GBs) exceeds L2", "execution": b["execution"], "seed": SEED},
            "back_to_back": n_all / (ms_s / 1e3), "back_to_back_ms_per_step": ms_s, "speedup": ms_s / ms_e,
            "branches": b["branches"], "steps_per_launch": b["steps_per_launch"],
            "gpu_launches": b["gpu_launches_per_step"] * b["steps"], "diagnostics_bit_identical": differs == 0.0,
            "clocks": {k: clocks.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons", "samples", "source")},
        }))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def ctypes_int(L, fn, handle):
    import ctypes as C
    v = C.c_int()
    getattr(L, fn)(C.c_void_p(handle), C.byref(v))
    return v.value


def e2e_run(cs, cfg, fluid, p, lo, hi, steps, device, stream, flush, warmup=3, arith=None):
    """Public-API run with host buffers: the state upload, then per step the
    frame-motion input (host->device) and the step's diagnostics
    (device->host), then the state download.  The diagnostics go through
    request_diagnostics / fetch_diagnostics as a control loop reads them: each
    step's record is requested after the step and read while the next step
    runs (the last one at the end of the last step).  Device-timed per step
    with L2 flushed between steps.  The same sequence runs once untimed first
    (`warmup` steps): the solver's device storage and step graphs are then in
    place, and the timed upload of the same-sized state reuses them, as a loop
    of runs on one Solver does."""
    import torch
    solver = cs.Solver(cfg, fluid, device)
    if arith is not None:
        solver.field_arithmetic = arith
    x = np.ascontiguousarray(p["position"], np.float64)
    arrays = [x, p["mass"].astype(np.float64), p["density"].astype(np.float64), p["temperature"].astype(np.float64)]
    state_in = sum(a.nbytes for a in arrays) + p["phase"].nbytes + p["normal"].nbytes + p["flags"].nbytes
    st = torch.cuda.ExternalStream(solver.stream_handle, device=device)

    def run(k_steps, ev=None, host=None):
        out = 0
        for k in range(k_steps):
            if ev is not None:
                flush.zero_()
                ev[k][0].record(st)
            t0 = time.perf_counter()
            if k == 0:
                load(solver, p, lo, hi)
            t1 = time.perf_counter()
            a = 0.01 * math.sin(0.01 * k)
            solver.set_frame_motion(acceleration=(a, 0.0, 0.0))
            solver.step()
            solver.request_diagnostics()
            if k > 0:  # the previous step's record
                _ = solver.fetch_diagnostics().slosh_force
            if k == k_steps - 1:  # and this one's, at the end
                _ = solver.fetch_diagnostics().slosh_force
            t2 = time.perf_counter()
            if k == k_steps - 1:
                parts = solver.particles()
                out = sum(v.nbytes for v in parts.values())
            t3 = time.perf_counter()
            if ev is not None:
                ev[k][1].record(st)
            if host is not None:
                host["upload_ms"] += (t1 - t0) * 1e3
                host["steps_ms"] += (t2 - t1) * 1e3
                host["download_ms"] += (t3 - t2) * 1e3
        return out

    with torch.cuda.stream(st):
        run(max(warmup, 1))
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    host = {"upload_ms": 0.0, "steps_ms": 0.0, "download_ms": 0.0}
    with torch.cuda.stream(st):
        state_out = run(steps, ev, host)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    n = solver.num_particles
    ctl = 3 * 4 * 4          # acceleration, omega, omega_dot, origin (float3 each)
    diag = 8 * 25 + 8 * 64   # diagnostics reduction + scalar block
    return {"value": n * steps / (ms / 1e3), "unit": UNIT,
            "h2d_bytes_per_step": int(state_in / steps + ctl), "d2h_bytes_per_step": int(diag + state_out / steps),
            "steps": steps, "host_wall_ms": {k: round(v, 3) for k, v in host.items()},
            "timing": "CUDA events per step (host work inside), L2 flushed between steps; one untimed run of the "
                      "same sequence first",
            "diagnostics": "every step's record read on the host: requested after the step, fetched while the next "
                           "step runs (request_diagnostics / fetch_diagnostics)"}


# SPHERIC Test 2 pressure sensors (validation/spheric_test2/run.py:30-33,69-73
# of the reference): four on the obstacle's front face, four on its top; then
# four on the floor along the column's path (x = 2.8, 2.2 under the column,
# 1.8, 1.6 where the front arrives), which the series reaches sooner.
def spheric_sensors(dx, floor=True):
    x_front, box_h, y = 0.744, 0.161, 0.403 / 2 - 0.176
    offs = (0.021, 0.061, 0.101, 0.141)
    pts = [(x_front + 0.5 * dx, y, z) for z in offs] + [(x_front - o, y, box_h + 0.5 * dx) for o in offs]
    if floor:
        pts += [(x, 0.0, 0.5 * dx) for x in (2.8, 2.2, 1.8, 1.6)]
    return np.array(pts, np.float32)


def probe_series_run(cs, device, dx, steps, arith):
    """The dam break's probe-pressure time series at the eight SPHERIC sensors,
    every step, against the reference's FP64 build on the same inputs (and its
    FP32 build, the single-precision noise floor).  The FP64 run's own time
    steps differ, so its series is interpolated linearly to this run's step
    times; a sample counts where both runs read the sensor wet.  Error per
    sensor: max |p - p64| / max |p64| over the wet samples."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refpy
    if not refpy.ref_available(fp64=True):
        return None
    label, cfg, fluid, p, lo, hi = workload("dam_break", cs, dx)
    s = cs.Solver(cfg, fluid, device)
    s.field_arithmetic = arith
    load(s, p, lo, hi)
    _, rcfg, rfluid, rp, rlo, rhi = ref_workload("dam_break", dx)
    refs = {}
    for name, fp64 in (("fp64", True), ("fp32", False)):
        r = refpy.Ref(rcfg, rfluid, fp64=fp64)
        r.set_threads(os.cpu_count() or 1)
        r.set_particles(rp, rlo, rhi)
        refs[name] = r
    pts = spheric_sensors(dx)
    series = {"ours": ([], []), "fp64": ([], []), "fp32": ([], [])}
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step()
        series["ours"][0].append(s.time)
        series["ours"][1].append(s.probe_pressure(pts))
        for name, r in refs.items():
            r.step(1)
            series[name][0].append(r.time()[0])
            series[name][1].append(r.probe_pressure(pts))
    wall = time.perf_counter() - t0

    def err(name):
        t, v = np.asarray(series[name][0]), np.asarray(series[name][1], np.float64)
        t64, v64 = np.asarray(series["fp64"][0]), np.asarray(series["fp64"][1], np.float64)
        out = []
        for k in range(len(pts)):
            ref_k = np.interp(t, t64, np.nan_to_num(v64[:, k], nan=np.inf))
            wet = np.isfinite(v[:, k]) & np.isfinite(ref_k) & (t <= t64[-1])
            if not wet.any():
                out.append(None)
                continue
            scale = max(float(np.abs(ref_k[wet]).max()), 1e-30)
            out.append(float(np.abs(v[wet, k] - ref_k[wet]).max() / scale))
        return out

    wet = np.isfinite(np.asarray(series["ours"][1])).mean(axis=0)
    return {"workload": label, "steps": steps,
            "sensors": "P1-P4 obstacle front face, P5-P8 obstacle top (run.py:69-73), F1-F4 floor at x = 2.8, 2.2, "
                       "1.8, 1.6 m",
            "field_arithmetic": "fast" if arith == cs.FieldArithmetic.Fast else "exact",
            "t_end": float(series["ours"][0][-1]), "wet_fraction": [float(w) for w in wet],
            "error_vs_fp64": err("ours"), "reference_fp32_error_vs_fp64": err("fp32"),
            "peak_pressure_fp64": [float(np.nanmax(np.asarray(series["fp64"][1])[:, k]))
                                   if np.isfinite(np.asarray(series["fp64"][1])[:, k]).any() else None
                                   for k in range(len(pts))],
            "wall_s": wall,
            "note": "error = max |p - p_fp64| / max |p_fp64| over the samples where both read the sensor wet; "
                    "the FP64 series interpolated to this run's step times"}


def side_force_run(cs, device, steps, arith, dx=None):
    """The LH2 sphere under its manoeuvre: a lateral (x) acceleration pulse of
    0.05 m/s^2 over the first 0.5 s, then a slew ramped to 5 deg/s about the
    tank centre (pitch, the y axis) over the next 0.5 s.  Every step the
    diagnostics give the slosh force; over the pulse the impulse on the tank
    is compared with -M a t (M the fluid mass), raw and corrected by the
    liquid's own momentum change in the tank frame (impulse balance: the walls
    take -M a t less what the liquid keeps as relative momentum)."""
    label, cfg, fluid, p, lo, hi = workload("c3", cs, dx)
    s = cs.Solver(cfg, fluid, device)
    s.field_arithmetic = arith
    load(s, p, lo, hi)
    a, t_pulse = 0.05, 0.5
    w = 5.0 * math.pi / 180.0
    times = [0.0, t_pulse, t_pulse + 1e-6, 2 * t_pulse]
    acc = np.array([[a, 0, 0], [a, 0, 0], [0, 0, 0], [0, 0, 0]], np.float64)
    omega = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [0, w, 0]], np.float64)
    s.set_maneuver(cs.ManeuverProfile(times, acc, omega, origin=(0.0, 0.0, 0.0)))
    d0 = s.diagnostics()
    M = d0.mass_liquid + d0.mass_vapor
    p0 = d0.liquid_momentum[0]
    impulse, t_in, p_in = 0.0, 0.0, p0
    rows = []
    t0 = time.perf_counter()
    for k in range(steps):
        s.step()
        d = s.diagnostics()
        if d.time <= t_pulse:
            impulse += d.dt * d.slosh_force[0]
            t_in, p_in = d.time, d.liquid_momentum[0]
        if k % max(1, steps // 50) == 0 or k == steps - 1:
            rows.append([round(d.time, 6), d.slosh_force[0], d.slosh_force[2], d.slosh_moment[1]])
    wall = time.perf_counter() - t0
    expect = -M * a * t_in
    return {"workload": label, "particles": int(s.num_particles), "steps": steps, "t_end": float(rows[-1][0]),
            "field_arithmetic": "fast" if arith == cs.FieldArithmetic.Fast else "exact",
            "fluid_mass": M, "pulse": {"a_x": a, "t": t_in, "impulse_x": impulse, "minus_M_a_t": expect,
                                       "ratio": impulse / expect,
                                       "ratio_momentum_corrected": (impulse + (p_in - p0)) / expect},
            "slew_deg_s": 5.0, "series_t_Fx_Fz_My": rows, "wall_s": wall}


def c5_solver(cs, device, dx=0.0034):
    """The differentiation workload: closed LN2 cylinder R 0.1 m, H
    0.25 m, dx 3.4 mm, fill 0.5, 2 K superheat, Lee 5 1/s both ways, 20 W
    heater, 1e-4 g; a fixed step of 1 ms and a pinned sound speed (0.5 m/s),
    and no splitting or merging inside the differentiated window."""
    fluid = cs.FluidProperties.liquid_nitrogen()
    cfg = cs.SolverConfig()
    cfg.dx = dx
    cfg.gravity = (0.0, 0.0, -9.81e-4)
    cfg.thermo_mode = cs.TankThermoMode.Closed
    cfg.heater_power = 20.0
    cfg.lee_evaporation = 5.0
    cfg.lee_condensation = 5.0
    cfg.fixed_dt = 1e-3
    cfg.sound_speed = 0.5
    cfg.split_ratio = 1e3
    cfg.merge_ratio = 0.0
    s = cs.Solver(cfg, fluid, device)
    fill = cs.FillSpec()
    fill.fill_fraction = 0.5
    fill.T_liquid = fluid.T_sat + 2.0
    s.build_tank(cs.CylinderTank(0.1, 0.25), fill)
    return s, fluid


def slab_run(cs, cfg, fluid, p, lo, hi, nslabs, devices, steps, label):
    """The workload as one tank cut along z into `nslabs` slabs of cell layers
    (CryoSPH.SlabSolver), against one Solver on the same inputs: wall clock
    per step with the device synchronised, the slab steps once as the
    captured group graph (the default) and once enqueued by host threads
    meeting at the exchange points; particle states compared bit for bit
    after the timed steps."""
    import torch
    one = cs.Solver(cfg, fluid, devices[0])
    load(one, p, lo, hi)
    runs = {"one_context": one}
    for name, graph in (("slabs", True), ("slabs_host_threads", False)):
        sl = cs.SlabSolver(cfg, fluid, slabs=nslabs, devices=devices)
        sl.graph_mode = graph
        sl.set_particles(p["position"], p["mass"], p["density"], p["temperature"], p["phase"], domain_lo=lo,
                         domain_hi=hi, normal=p["normal"], flags=p["flags"])
        runs[name] = sl
    times = {}
    for name, obj in runs.items():
        obj.run_steps(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        obj.run_steps(steps)
        torch.cuda.synchronize()
        times[name] = (time.perf_counter() - t0) / steps * 1e3
    a = one.particles()
    same = {name: all(np.array_equal(np.asarray(a[k]), np.asarray(b[k])) for k in a)
            for name, b in ((n, runs[n].particles()) for n in ("slabs", "slabs_host_threads"))}
    sl = runs["slabs"]
    lay = sl.layout()
    return {"workload": label, "slabs": nslabs, "devices": devices, "steps": steps,
            "ms_per_step": times["slabs"], "graph_mode": sl.graph_mode,
            "host_threads_ms_per_step": times["slabs_host_threads"],
            "one_context_ms_per_step": times["one_context"],
            "z_begin": list(lay["z_begin"]), "owned": list(lay["owned"]), "held": list(lay["held"]),
            "ghost_fraction": sum(lay["held"]) / max(sum(lay["owned"]), 1) - 1.0,
            "bit_identical": bool(same["slabs"] and same["slabs_host_threads"]),
            "timing": "wall clock, device synchronised"}


def adjoint_run(cs, device, steps, every, knots=16):
    """The LN2 boil-off window: gradients of the time-integrated slosh force and
    moment and the final ullage pressure with respect to the surface tension,
    the contact angle, the Lee coefficient and 16 piecewise-constant lateral
    frame-acceleration knots (seeded U[-0.05, 0.05] m/s^2), through the
    torch.autograd.Function over the hand-written adjoint.  Wall-clock times
    with the device synchronised: the plain forward (the same steps, step
    graphs, no checkpoints), the differentiated forward (checkpoints every
    `every` steps) and the backward (segment recomputation + reverse passes)."""
    import torch
    import cryo_adjoint as ca
    free0 = torch.cuda.mem_get_info(device)[0]
    knots = min(knots, steps)
    s, fluid = c5_solver(cs, device)
    s.run_steps(3)
    blob = s.save_state()
    rng = np.random.Generator(np.random.PCG64(SEED))
    kn = np.zeros((knots, 3))
    kn[:, 0] = rng.uniform(-0.05, 0.05, knots)
    dt = float(s.config.fixed_dt)
    times, _ = ca.knot_schedule(s.time, dt, steps, knots)
    s.set_maneuver(ca._maneuver(times, kn))
    s.run_steps(1)  # graph capture outside the timing
    # one untimed window first: the window's device arena is allocated once
    # and reused by later windows of the same size (an optimisation loop)
    s.load_state(blob)
    s.adjoint_forward(steps, every)
    s.adjoint_backward([1.0] * 7)
    s.load_state(blob)
    s.set_maneuver(ca._maneuver(times, kn))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.run_steps(steps)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    s.load_state(blob)
    sigma = torch.tensor(float(fluid.sigma), dtype=torch.float64, requires_grad=True)
    theta = torch.tensor(float(s.config.contact_angle_deg), dtype=torch.float64, requires_grad=True)
    lee = torch.tensor(5.0, dtype=torch.float64, requires_grad=True)
    kt = torch.tensor(kn, dtype=torch.float64, requires_grad=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = ca.slosh_window(s, sigma, theta, lee, kt, steps, every)
    torch.cuda.synchronize()
    t_fwd = time.perf_counter() - t0
    weights = torch.tensor([1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1e-4], dtype=torch.float64)
    loss = (out * weights).sum()
    t0 = time.perf_counter()
    loss.backward()
    torch.cuda.synchronize()
    t_bwd = time.perf_counter() - t0
    used = free0 - torch.cuda.mem_get_info(device)[0]
    # full-size check: Richardson-extrapolated central differences of the
    # same loss through the forward (this library's FP32 steps); steps h and
    # h/2 with h = 2e-2 of the value (knots: 2e-3 m/s^2); "fd_spread" is
    # |D(h) - D(h/2)| / |R|, the size of the differences' own error
    def loss_at(sig=None, th=None, le=None, kk=None):
        s.load_state(blob)
        with torch.no_grad():
            o = ca.slosh_window(s, float(sigma) if sig is None else sig, float(theta) if th is None else th,
                                float(lee) if le is None else le, kn if kk is None else kk, steps, every)
        return float((o * weights).sum())

    def knot_loss(kidx, v):
        kk = kn.copy()
        kk[kidx, 0] = v
        return loss_at(kk=kk)

    probes = [("lee", float(lee), 2e-2 * float(lee), lambda v: loss_at(le=v)),
              ("contact_angle_deg", float(theta), 2e-2 * float(theta), lambda v: loss_at(th=v))]
    probes += [(f"knot{k}_x", float(kn[k, 0]), 2e-3, (lambda kidx: lambda v: knot_loss(kidx, v))(k))
               for k in (0, knots // 2)]
    ad = {"lee": float(lee.grad), "contact_angle_deg": float(theta.grad),
          **{f"knot{k}_x": float(kt.grad[k, 0]) for k in (0, knots // 2)}}
    check = {}
    for name, base, h, get in probes:
        d1 = (get(base + h) - get(base - h)) / (2 * h)
        d2 = (get(base + h / 2) - get(base - h / 2)) / h
        r = (4 * d2 - d1) / 3
        check[name] = {"adjoint": ad[name], "fd": r, "rel": abs(ad[name] - r) / max(abs(r), 1e-300),
                       "fd_spread": abs(d1 - d2) / max(abs(r), 1e-300)}
    res = {
        "workload": "c5_ln2_boiloff_cylinder_dx0.0034", "particles": int(s.num_particles), "steps": steps,
        "checkpoint_every": every, "knots": knots,
        "plain_forward_s": t_plain, "adjoint_forward_s": t_fwd, "backward_s": t_bwd,
        "adjoint_forward_ratio": (t_fwd + t_bwd) / t_plain,
        "backward_over_forward": t_bwd / t_plain,
        "window_device_bytes": int(s.adjoint_memory), "process_device_bytes": int(used),
        "objectives": [float(v) for v in out.detach()],
        "grad": {"sigma": float(sigma.grad), "contact_angle_deg": float(theta.grad), "lee": float(lee.grad),
                 "knots_x": [float(v) for v in kt.grad[:, 0]]},
        "loss": "sum of int F, int M (N s, N m s) + 1e-4 p_ullage (Pa)",
        "fd_check": check,
        "fd_note": "Richardson-extrapolated central differences of the FP32 forward over the same window",
        "timing": "wall clock, device synchronised, after one untimed window (arena allocated); plain forward = "
                  "the same steps through Solver.run_steps",
    }
    s.adjoint_release()
    return res


def _ref_structs(cs_cfg, fluid):
    """The reference driver's config and fluid structs from module objects."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref_abi
    kw = {}
    for name, _ in ref_abi.Config._fields_:
        v = getattr(cs_cfg, name)
        kw[name] = tuple(v) if name == "gravity" else (int(v.value) if hasattr(v, "value") else
                                                      (int(v) if isinstance(v, bool) else v))
    f = ref_abi.Fluid()
    for k, _ in ref_abi.Fluid._fields_:
        setattr(f, k, getattr(fluid, k))
    return ref_abi.config(**kw), f


def adjoint_fd64_run(cs, device, steps, every, knots=4):
    """The LN2 boil-off window from its initial lattice: this library's adjoint
    gradients (FP32 forward, hand-written reverse passes) against central
    differences of the same loss through the reference's FP64 forward
    (oracle/_ref/libcryoref64.so, every host thread), for the contact angle,
    the Lee coefficient and the first manoeuvre knot.  The FP64 forward has no
    single-precision noise, so a small step (1e-3 relative; 1e-4 m/s^2 for the
    knot) gives a clean difference quotient."""
    import torch
    import cryo_adjoint as ca
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import refpy
    if not refpy.ref_available(fp64=True):
        return None
    s, fluid = c5_solver(cs, device)
    p = s.particles()
    lo, hi = cs.tank_domain(cs.CylinderTank(0.1, 0.25), float(s.config.dx), 3)
    # Initialise with the base parameters (the initial rate evaluation, whose
    # accelerations the first half-kick uses, is not part of the window);
    # the reference below is initialised the same way before its perturbation.
    s.next_dt()
    dt = float(s.config.fixed_dt)
    rng = np.random.Generator(np.random.PCG64(SEED))
    kn = np.zeros((knots, 3))
    kn[:, 0] = rng.uniform(-0.05, 0.05, knots)
    times, _ = ca.knot_schedule(0.0, dt, steps, knots)
    weights = np.array([1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1e-4])
    theta0, lee0 = float(s.config.contact_angle_deg), 5.0
    # adjoint
    th = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    le = torch.tensor(lee0, dtype=torch.float64, requires_grad=True)
    kt = torch.tensor(kn, dtype=torch.float64, requires_grad=True)
    t0 = time.perf_counter()
    out = ca.slosh_window(s, float(fluid.sigma), th, le, kt, steps, every)
    (out * torch.tensor(weights)).sum().backward()
    t_adj = time.perf_counter() - t0
    ad = {"contact_angle_deg": float(th.grad), "lee": float(le.grad), "knot0_x": float(kt.grad[0, 0])}
    base_cfg, base_fluid = _ref_structs(s.config, fluid)
    arrays = {"x": p["position"], "v": p["velocity"], "m": p["mass"], "rho": p["density"], "T": p["temperature"],
              "phase": p["phase"], "nrm": p["normal"], "flags": p["flags"]}

    def loss64(theta=theta0, lee=lee0, knot0=kn[0, 0]):
        cfg = type(base_cfg).from_buffer_copy(base_cfg)
        cfg.lee_evaporation = cfg.lee_condensation = lee  # not read by the initialisation
        r = refpy.Ref(cfg, base_fluid, fp64=True)
        r.set_threads(os.cpu_count() or 1)
        r.set_particles(arrays, lo, hi)
        r.next_dt()  # initialised with the base contact angle and no frame motion
        r.set_contact_angle(theta)
        k = kn.copy()
        k[0, 0] = knot0
        r.set_maneuver(times, np.repeat(k, 2, axis=0))
        obj = np.zeros(7)
        for _ in range(steps):
            r.step(1)
            d = r.diagnostics()
            obj[:3] += dt * np.asarray(d.slosh_force, np.float64)
            obj[3:6] += dt * np.asarray(d.slosh_moment, np.float64)
        obj[6] = r.diagnostics().p_ullage
        r.close()
        return float(obj @ weights)

    t0 = time.perf_counter()
    check = {}
    for name, base, h, call in (("contact_angle_deg", theta0, 1e-3 * theta0, lambda v: loss64(theta=v)),
                                ("lee", lee0, 1e-3 * lee0, lambda v: loss64(lee=v)),
                                ("knot0_x", float(kn[0, 0]), 1e-4, lambda v: loss64(knot0=v))):
        fd = (call(base + h) - call(base - h)) / (2 * h)
        check[name] = {"adjoint": ad[name], "fd64": fd, "rel": abs(ad[name] - fd) / max(abs(fd), 1e-300)}
    s.adjoint_release()
    return {"workload": "c5_ln2_boiloff_cylinder_dx0.0034", "window_steps": steps, "checkpoint_every": every,
            "knots": knots, "start": "initial lattice (t = 0), initialised with the base parameters",
            "fd_check_fp64": check,
            "loss": "sum of int F, int M (N s, N m s) + 1e-4 p_ullage (Pa)",
            "adjoint_s": t_adj, "fd64_s": time.perf_counter() - t0}


def batched_run(cs, tanks, steps, warmup, device, tune_steps=3, arith=None):
    """The 64-tank ensemble: the tanks advanced together by one cs.Ensemble (one
    graph launch per ensemble step, branch count autotuned) against the same
    tanks stepped back to back by plain Solvers.  Both sides take the same
    total number of steps, so every tank's diagnostics can be compared bit for
    bit at the end.  Device time from CUDA events; the ensemble's state
    (hundreds of MB) exceeds L2, the back-to-back tanks are each L2-sized (an
    advantage to the back-to-back side)."""
    import torch

    def make():
        out = []
        for tk in tanks:
            sv = cs.Solver(tk["cfg"], tk["fluid"], device)
            if arith is not None:
                sv.field_arithmetic = arith
            load(sv, tk["p"], tk["lo"], tk["hi"])
            sv.set_maneuver(tk["maneuver"])
            out.append(sv)
        return out

    ens_tanks = make()
    ens = cs.Ensemble(device)
    for sv in ens_tanks:
        ens.add(sv)
    cands = sorted({k for k in (len(tanks), 32, 16, 8, 4) if 1 <= k <= len(tanks)}, reverse=True)
    branches, per_launch, _ = ens.tune(cands, [1, 2, 4], tune_steps, [1, 2, 4])
    ens.run_steps(warmup)
    before = ens_tanks[0].step_count
    ms_ens = ens.step_time(steps)
    timed_steps = ens_tanks[0].step_count - before - per_launch  # step_time's untimed launch excluded
    total_steps = ens_tanks[0].step_count
    n_total = sum(tk["n"] for tk in tanks)
    launches = ens.launches_per_step
    tile = ens.tile
    d_ens = [d.as_dict() for d in ens.diagnostics()]
    del ens

    solo = make()
    ms_solo = 0.0
    for sv in solo:
        sv.run_steps(total_steps - timed_steps)
        st = torch.cuda.ExternalStream(sv.stream_handle, device=device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        sv.run_steps(timed_steps)
        b.record(st)
        b.synchronize()
        ms_solo += a.elapsed_time(b)
    d_solo = [sv.diagnostics().as_dict() for sv in solo]
    same = all(json.dumps(x, sort_keys=True) == json.dumps(y, sort_keys=True) for x, y in zip(d_ens, d_solo))
    return {
        "workload": f"c4_ensemble_{len(tanks)}_tanks", "tanks": len(tanks), "particles": n_total,
        "particles_min": min(tk["n"] for tk in tanks), "particles_max": max(tk["n"] for tk in tanks),
        "steps": timed_steps, "value": n_total / (ms_ens / 1e3) if ms_ens > 0 else None, "unit": UNIT,
        "ms_per_step": ms_ens, "back_to_back": n_total * timed_steps / (ms_solo / 1e3),
        "back_to_back_ms_per_step": ms_solo / timed_steps,
        "speedup": (ms_solo / timed_steps) / ms_ens if ms_ens > 0 else None, "branches": branches,
        "steps_per_launch": per_launch, "tile": tile,
        "gpu_launches_per_step": launches, "diagnostics_bit_identical": bool(same),
        "execution": "CUDA graph launches of steps_per_launch ensemble steps (every tank's kernels as concurrent branches)",
    }


def roofline(cs, cabi, L, cfg, fluid, p, lo, hi, steps, n_fluid, n_wall, has_vapor, label, arith=None):
    import ctypes as C
    import cryo_roofline as RF
    solver = cs.Solver(cfg, fluid)
    if arith is not None:
        solver.field_arithmetic = arith
    load(solver, p, lo, hi)
    solver.run_steps(3)
    h = C.c_void_p(solver.handle)
    L.cryo_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.cryo_kernel_times.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_char_p, C.POINTER(C.c_double),
                                    C.POINTER(C.c_longlong)]
    L.cryo_set_profiling(h, 1)
    solver.run_steps(steps)
    cnt = C.c_int(0)
    L.cryo_kernel_times(h, C.byref(cnt), None, None, None)
    k = cnt.value
    names = C.create_string_buffer(64 * k)
    ms = (C.c_double * k)()
    launches = (C.c_longlong * k)()
    cnt2 = C.c_int(k)
    L.cryo_kernel_times(h, C.byref(cnt2), names, ms, launches)
    L.cryo_set_profiling(h, 0)
    rows = []
    for i in range(k):
        nm = names.raw[64 * i: 64 * i + 64].split(b"\0")[0].decode()
        rows.append((nm, ms[i], launches[i]))
    total = sum(r[1] for r in rows)
    top = max(rows, key=lambda r: r[1])
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    nc = 0
    avg_ms = top[1] / max(top[2], 1)
    alg = RF.kernel_bytes(top[0], cfg_dict(cfg), n_fluid, n_wall, has_vapor, nc)
    achieved = alg / (avg_ms / 1e3) / 1e9
    traffic = ncu_traffic(top[0], label)
    return {"kernel": top[0], "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "traffic_cold": ncu_traffic(top[0], label, cold=True),
            "traffic_note": "DRAM bytes per launch from one ncu launch list of this command with the L2 as the timed "
                            "steps leave it (--cache-control none; flushed between steps only); traffic_cold: the "
                            "same with the L2 flushed before the kernel",
            "ncu_utilisation": ncu_utilisation(top[0], label),
            "algorithmic_bytes": alg, "avg_launch_ms": avg_ms,
            "share": top[1] / total if total else None, "peak_source": "measured" if peaks else "fallback",
            "kernels": {r[0]: {"ms_per_step": r[1] / steps, "launches": r[2]} for r in sorted(rows, key=lambda r: -r[1])}}


def cfg_dict(cfg):
    out = {}
    for k in ["density_mode", "transport_velocity", "thermal", "phase_change", "surface_tension", "wetting_model",
              "sps_turbulence", "transport_stress"]:
        v = getattr(cfg, k)
        out[k] = int(v.value) if hasattr(v, "value") else int(v)
    return out


def ncu_utilisation(kernel, label):
    """Issue-slot, FMA-pipe, L1 and DRAM utilisation of `kernel` from the
    committed ncu capture (the neighbour passes are bound by issue and
    latency, not HBM; null if absent)."""
    try:
        with open(os.path.join(REPO, "profiles", "ncu_dram.json")) as fh:
            return json.load(fh).get("utilisation", {}).get(label, {}).get(kernel)
    except (OSError, ValueError):
        return None


def ncu_traffic(kernel, label, cold=False):
    """DRAM bytes per launch of `kernel` in the step (L2 as the timed steps leave it; cold=True: L2 flushed
    before the kernel) from the committed ncu launch list (null if absent)."""
    path = os.path.join(REPO, "profiles", "ncu_dram.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        e = (d.get("cold", {}) if cold else d).get(label, {}).get(kernel)
        return None if e is None else float(e)
    except (OSError, ValueError):
        return None


if __name__ == "__main__":
    sys.exit(main())
