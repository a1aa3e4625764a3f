"""Batched ensemble (cs.Ensemble over cryo_ensemble_*): every member's state
after N ensemble steps must equal, bit for bit, the same tank stepped N times
alone by the plain path -- whatever the branch count, after tuning, after a
member was stepped on its own in between, and after a member left."""
import json
import os
import sys

import numpy as np
import pytest

import CryoSPH as cs

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
import bench  # noqa: E402  (the config-4 tank generator)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tanks():
    return bench.c4_tanks(cs, count=6, n_lo=2_000, n_hi=15_000, seed=7)


def solvers(tanks):
    out = []
    for tk in tanks:
        s = cs.Solver(tk["cfg"], tk["fluid"], 0)
        bench.load(s, tk["p"], tk["lo"], tk["hi"])
        s.set_maneuver(tk["maneuver"])
        out.append(s)
    return out


def same_state(a, b):
    pa, pb = a.particles(), b.particles()
    for k in pa:
        if not np.array_equal(np.asarray(pa[k]).view(np.uint8), np.asarray(pb[k]).view(np.uint8)):
            return f"particles.{k}"
    da, db = a.diagnostics().as_dict(), b.diagnostics().as_dict()
    if json.dumps(da, sort_keys=True) != json.dumps(db, sort_keys=True):
        return "diagnostics"
    return None


def test_ensemble_steps_equal_solo_steps_bitwise(cuda_device, tanks):
    ens_s, solo = solvers(tanks), solvers(tanks)
    ens = cs.Ensemble(0)
    for s in ens_s:
        ens.add(s)
    assert len(ens) == len(tanks)
    ens.run_steps(20)
    for s in solo:
        s.run_steps(20)
    for k, (a, b) in enumerate(zip(ens_s, solo)):
        assert a.step_count == 20
        assert same_state(a, b) is None, (k, same_state(a, b))
    assert ens.launches_per_step > 0


@pytest.mark.parametrize("chains", [1, 2, 0])
def test_branch_counts_and_tuning_keep_bit_identity(cuda_device, tanks, chains):
    ens_s, solo = solvers(tanks), solvers(tanks)
    ens = cs.Ensemble(0)
    for s in ens_s:
        ens.add(s)
    ens.chains = chains
    ens.run_steps(4)
    best, per, ms = ens.tune([len(tanks), 3, 1], [1, 2], 2)
    assert best in (len(tanks), 3, 1) and per in (1, 2) and ms > 0
    ens.steps_per_launch = 4
    ens.run_steps(7)  # one 4-step launch, then single steps
    total = ens_s[0].step_count
    assert all(s.step_count == total for s in ens_s)
    for s in solo:
        s.run_steps(total)
    for k, (a, b) in enumerate(zip(ens_s, solo)):
        assert same_state(a, b) is None, (k, same_state(a, b))


@pytest.mark.parametrize("per_launch", [2, 4])
def test_multi_step_launches_from_either_parity(cuda_device, tanks, per_launch):
    """Launches of several steps, entered after an odd and after an even
    number of steps (both ping-pong parities), and a remainder of single steps."""
    ens_s, solo = solvers(tanks), solvers(tanks)
    ens = cs.Ensemble(0)
    for s in ens_s:
        ens.add(s)
    ens.steps_per_launch = per_launch
    ens.run_steps(1)
    ens.run_steps(2 * per_launch + 1)
    ens.run_steps(per_launch)
    n = 1 + 2 * per_launch + 1 + per_launch
    for s in solo:
        s.run_steps(n)
    for k, (a, b) in enumerate(zip(ens_s, solo)):
        assert a.step_count == n
        assert same_state(a, b) is None, (k, same_state(a, b))


def test_member_stepped_alone_and_removed(cuda_device, tanks):
    ens_s, solo = solvers(tanks), solvers(tanks)
    ens = cs.Ensemble(0)
    for s in ens_s:
        ens.add(s)
    ens.run_steps(3)
    ens_s[0].run_steps(1)          # parity of one member flips: the ensemble rebuilds
    ens_s[1].set_heater_power(5.0)  # a control change between ensemble steps
    ens.run_steps(3)
    ens.remove(ens_s[2])
    assert len(ens) == len(tanks) - 1
    ens.run_steps(2)
    counts = [3 + 1 + 3 + 2, 3 + 3 + 2, 3 + 3] + [3 + 3 + 2] * (len(tanks) - 3)
    solo[1].run_steps(3)
    solo[1].set_heater_power(5.0)
    solo[1].run_steps(5)
    for k, (s, n) in enumerate(zip(solo, counts)):
        if k != 1:
            s.run_steps(n)
    for k, (a, b) in enumerate(zip(ens_s, solo)):
        assert a.step_count == counts[k]
        assert same_state(a, b) is None, (k, same_state(a, b))


def test_bad_members_are_refused(cuda_device, tanks):
    ens = cs.Ensemble(0)
    empty = cs.Solver(tanks[0]["cfg"], tanks[0]["fluid"], 0)
    with pytest.raises(ValueError):
        ens.add(empty)  # no particles
    s = solvers(tanks[:1])[0]
    ens.add(s)
    with pytest.raises(ValueError):
        ens.add(s)  # already a member
    other = cs.Ensemble(0)
    with pytest.raises(ValueError):
        other.add(s)  # member of another ensemble
    with pytest.raises(ValueError):
        ens.chains = -1
    with pytest.raises(ValueError):
        ens.steps_per_launch = 3


@pytest.mark.parametrize("tile", [2, 4])
def test_member_tiles_keep_bit_identity(cuda_device, tanks, tile):
    """The members' tile (particles per thread of their grid-stride kernels)
    changes launch grids only: results equal the solo steps bit for bit,
    and the tuner's tile axis picks one of its candidates."""
    ens_s, solo = solvers(tanks), solvers(tanks)
    ens = cs.Ensemble(0)
    for s in ens_s:
        ens.add(s)
    ens.tile = tile
    assert ens.tile == tile
    ens.run_steps(6)
    best, per, ms = ens.tune([len(tanks)], [1], 2, [1, tile])
    assert ens.tile in (1, tile) and ms > 0
    ens.run_steps(3)
    total = ens_s[0].step_count
    for s in solo:
        s.run_steps(total)
    for k, (a, b) in enumerate(zip(ens_s, solo)):
        assert same_state(a, b) is None, (k, same_state(a, b))
    with pytest.raises(ValueError):
        ens.tile = 0
