"""The algorithmic-byte model behind bench.py's roofline (cryo_roofline.py).

`roofline.achieved` in the bench line is the force pass's algorithmic bytes
per launch divided by its measured launch time, so the per-particle figures
are part of the reported number.  These CPU tests pin them for the dam break
(SPHERIC T2, dx 0.02 m: continuity density, no surface tension, no heat, no
phase change), check the dam break's particle counts that turn them into
bytes per launch, and check that the switches of a two-phase tank add the
fields those passes then read."""
import os
import sys

import pytest

import cryo_roofline as rf

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
import bench  # noqa: E402

# (fluid bytes, wall bytes) per particle and launch on the dam break
DAM_BREAK = {
    "k_kick_drift_keys": (101, 17),
    "k_gather": (144, 144),
    "k_density": (37, 9),
    "k_wall": (1, 53),
    "k_interface": (49, 1),
    "k_forces": (117, 53),
    "k_kick": (37, 1),
    "k_saturation": (9, 1),
}
N_FLUID, N_WALL = 82_350, 121_312


@pytest.mark.parametrize("kernel", sorted(DAM_BREAK))
def test_dam_break_bytes_per_particle(kernel):
    cfg = bench.workload_spec("dam_break")["config"]
    assert rf.per_particle(kernel, cfg, False) == DAM_BREAK[kernel]


def test_dam_break_force_pass_bytes_per_launch():
    cfg = bench.workload_spec("dam_break")["config"]
    assert rf.kernel_bytes("k_forces", cfg, N_FLUID, N_WALL, False) == 117 * N_FLUID + 53 * N_WALL == 16_064_486


def test_dam_break_particle_counts():
    import CryoSPH as cs
    _, _, _, p, _, _ = bench.workload("dam_break", cs)
    phase = p["phase"]
    assert int((phase == 2).sum()) == N_WALL
    assert int((phase != 2).sum()) == N_FLUID


def test_two_phase_switches_add_fields():
    dam = bench.workload_spec("dam_break")["config"]
    two = dict(dam, surface_tension=1, thermal=1, phase_change=1)
    for kernel in ("k_forces", "k_interface", "k_kick"):
        f_dam, _ = rf.per_particle(kernel, dam, False)
        f_two, _ = rf.per_particle(kernel, two, True)
        assert f_two > f_dam, kernel


def test_unknown_kernel_and_sort_passes():
    assert rf.per_particle("k_not_a_kernel", {}, False) == (0, 0)
    assert rf.kernel_bytes("k_cells", {}, 0, 0, False, num_cells=99) == 4 * 100
    assert rf.sort_passes(1) == 1
    assert rf.sort_passes(255) == 1
    assert rf.sort_passes(256) == 2
    assert rf.sort_passes(65_535) == 2
    assert rf.sort_passes(65_536) == 3
