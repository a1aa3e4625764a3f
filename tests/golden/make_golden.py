"""Generates the golden vectors in this directory from the reference's own CPU
build (oracle/_ref/libcryoref.so, compiled from the reference sources by
oracle/Makefile), run with one OpenMP thread so sums are in index order.

  python tests/golden/make_golden.py

Fixtures (numpy .npz, small):
  box_split.npz   closed LN2 box with superheat and a low split ratio: the
                  jittered input, and after 1 and 200 steps every per-particle
                  field plus the diagnostics (splits start near step 190)
  c1_pass.npz     the LN2 cylinder (R 0.05 m, dx 4 mm): input, then after the first grid build the
                  cell tables and neighbour counts/id sums (neighbor_stats,
                  spatial_hash.cu:140-171)
  cloud.npz       a random cloud (3000 points, seed 7, radius 0.08) as in
                  test_spatial_hash.cpp:25-51: sorted state and the neighbour
                  counts / id sums of the reference's cell lists
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "tests"), os.path.join(REPO, "oracle"),
                os.path.join(REPO, "microgravity-cryogenic-multi-phase-sph-solver_b200")]

import cryo_cabi as cabi  # noqa: E402
import refpy  # noqa: E402
import scenarios as S  # noqa: E402

DIAG_KEYS = ["n_total", "n_liquid", "n_vapor", "n_wall", "mass_liquid", "mass_vapor", "mass_total", "kinetic_energy",
             "enthalpy", "heat_input", "evaporated_mass", "condensed_mass", "T_sat", "p_ullage", "max_speed",
             "splits", "merges", "time", "dt"]


def state(r, tag):
    out = {}
    for f in cabi.FIELDS:
        out[f"{tag}_{f}"] = r.field(f)
    d = r.diagnostics().as_dict()
    for k in DIAG_KEYS:
        out[f"{tag}_diag_{k}"] = np.array(d[k])
    out[f"{tag}_diag_slosh_force"] = np.array(d["slosh_force"])
    return out


def inputs(parts, lo, hi):
    return {"in_" + k: np.asarray(v) for k, v in parts.items()} | {"in_lo": np.array(lo), "in_hi": np.array(hi)}


def main():
    assert refpy.ref_available(), "build the reference first: make -C oracle ref"
    # box_split
    cfg, fl, parts, lo, hi = S.box_split()
    r = refpy.Ref(cfg, fl)
    r.set_threads(1)
    r.set_particles(parts, lo, hi)
    out = inputs(parts, lo, hi)
    r.step(1)
    out |= state(r, "s1")
    r.step(199)
    out |= state(r, "s200")
    np.savez_compressed(os.path.join(HERE, "box_split.npz"), **out)

    # c1 grid + neighbour stats
    cfg, fl, parts, lo, hi = S.c1()
    r = refpy.Ref(cfg, fl)
    r.set_threads(1)
    r.set_particles(parts, lo, hi)
    r.run_pass("grid_build")
    cs, ce = r.cell_tables()
    counts, lists = r.neighbor_lists()
    out = inputs(parts, lo, hi) | {"cell_start": cs, "cell_end": ce, "nbr_counts": counts,
                                   "nbr_checksum": np.array(np.sum(lists.astype(np.int64) * (np.arange(len(lists)) % 7 + 1))),
                                   "sorted_id": r.field("id"), "sorted_x": r.field("x")}
    np.savez_compressed(os.path.join(HERE, "c1_pass.npz"), **out)

    # random cloud (test_spatial_hash.cpp:14-51)
    rng = np.random.default_rng(7)
    n = 3000
    x = rng.random((n, 3)).astype(np.float32)
    arrays = {"x": x, "v": x[:, [2, 0, 1]].copy(), "m": (1.0 + x[:, 0]).astype(np.float32),
              "rho": np.full(n, 1000, np.float32), "T": (20.0 + x[:, 1]).astype(np.float32),
              "phase": np.where(np.arange(n) % 3 == 0, 1, 0).astype(np.uint8)}
    radius = 0.08
    c = cabi.py_config(dx=radius / 2.6, thermal=0, phase_change=0, surface_tension=0, velocity_scale=1.0)
    r = refpy.Ref(c, cabi.py_fluid(cabi.FLUID_LN2))
    r.set_particles(arrays, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    r.run_pass("grid_build")
    cnt, ids = r.neighbor_stats(radius)
    np.savez_compressed(os.path.join(HERE, "cloud.npz"), **{"in_" + k: v for k, v in arrays.items()},
                        radius=np.array(radius), counts=cnt, id_sums=ids, sorted_id=r.field("id"),
                        sorted_x=r.field("x"))
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
