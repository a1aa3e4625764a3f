"""Host-side pieces of the slab decomposition (cryo_slabs_*), no GPU:

* the layer partition (cryo_slab_partition);
* a model of the ownership and ordering rules in numpy: slabs that refresh
  from their neighbours' facing layers between steps, sort stably by cell
  key and append split children, hold in their owned layers (and in the
  ghost layer next to them) exactly the particles, in exactly the order, of
  the whole tank's sorted arrays.  This is the property the device code
  relies on for bit-identical results."""
import numpy as np
import pytest

import cryo_cabi as cabi

DEPTH = 2  # layers a slab copies from each neighbour between steps


def test_partition_balances_counts():
    counts = np.array([0, 5, 40, 40, 40, 40, 40, 40, 40, 40, 5, 0])
    zb = cabi.slab_partition(counts, 3, min_layers=2)
    assert zb[0] == 0 and zb[-1] == len(counts)
    assert np.all(np.diff(zb) >= 2)
    owned = [counts[zb[r]:zb[r + 1]].sum() for r in range(3)]
    assert sum(owned) == counts.sum()
    assert max(owned) - min(owned) <= 2 * counts.max()


def test_partition_keeps_min_layers():
    counts = np.zeros(12, np.int64)
    counts[0] = 1000  # everything in one layer
    zb = cabi.slab_partition(counts, 4, min_layers=3)
    assert zb.tolist() == [0, 3, 6, 9, 12]


def test_partition_single_slab():
    zb = cabi.slab_partition(np.ones(7, np.int64), 1, min_layers=3)
    assert zb.tolist() == [0, 7]


@pytest.mark.parametrize("args", [(np.ones(8, np.int64), 3, 3), (np.ones(8, np.int64), 0, 1),
                                  (np.ones(8, np.int64), 2, 0), (-np.ones(8, np.int64), 2, 1)])
def test_partition_rejects(args):
    with pytest.raises(cabi.CryoError):
        cabi.slab_partition(args[0], args[1], min_layers=args[2])


# ---------------------------------------------------------------- the model
NZ, NXY = 16, 5  # layers, cells per layer


def key_of(z, c):
    return z * NXY + c


class Tank:
    """Particle ids in array order, with each id's cell; a step moves every
    particle by at most one layer (the CFL bound), sorts stably by key, then
    lets some owned particles split (children appended) or die."""

    def __init__(self, rng, n):
        self.z = {i: int(rng.integers(0, NZ)) for i in range(n)}
        self.c = {i: int(rng.integers(0, NXY)) for i in range(n)}
        self.dead = set()
        self.next_id = n

    def key(self, i):
        return NZ * NXY if i in self.dead else key_of(self.z[i], self.c[i])


def drift(tank, rng, ids):
    for i in ids:
        if i in tank.dead:
            continue
        tank.z[i] = int(np.clip(tank.z[i] + rng.integers(-1, 2), 0, NZ - 1))
        tank.c[i] = int(rng.integers(0, NXY))


def stable_sort(tank, arr):
    keys = np.array([tank.key(i) for i in arr])
    order = np.argsort(keys, kind="stable")
    out = [arr[k] for k in order if keys[k] < NZ * NXY]
    return out


def layer_slice(tank, arr, z0, z1):
    return [i for i in arr if z0 <= tank.z[i] < z1]


@pytest.mark.parametrize("nslabs", [2, 3, 4])
def test_slab_orders_match_whole_tank(nslabs):
    run_model(nslabs, DEPTH)


def test_one_refresh_layer_is_not_enough():
    """With one refresh layer a particle that drifts from the second layer
    into the ghost layer is missing there: the model must notice."""
    with pytest.raises(AssertionError):
        run_model(3, 1)


def run_model(nslabs, DEPTH):
    rng = np.random.Generator(np.random.PCG64(7))
    tank = Tank(rng, 400)
    zb = [0] + [NZ * r // nslabs for r in range(1, nslabs)] + [NZ]
    # initial arrays: input order, each slab its layers +- DEPTH
    whole = list(range(400))
    slab = [[i for i in whole if zb[r] - DEPTH <= tank.z[i] < zb[r + 1] + DEPTH] for r in range(nslabs)]
    whole = stable_sort(tank, whole)
    slab = [stable_sort(tank, a) for a in slab]
    children = [[] for _ in range(nslabs)]
    whole_children = []
    for step in range(30):
        # ---- refresh (slabs) from the end-of-step layout
        own = [layer_slice(tank, slab[r], zb[r], zb[r + 1]) for r in range(nslabs)]
        new = []
        for r in range(nslabs):
            lo = layer_slice(tank, slab[r - 1], zb[r] - DEPTH, zb[r]) if r > 0 else []
            up = layer_slice(tank, slab[r + 1], zb[r + 1], zb[r + 1] + DEPTH) if r + 1 < nslabs else []
            lo_c = children[r - 1] if r > 0 else []
            up_c = children[r + 1] if r + 1 < nslabs else []
            new.append(lo + own[r] + up + lo_c + children[r] + up_c)
        slab = new
        whole = whole + whole_children
        # ---- one step: drift (the same motion everywhere), sort
        drift(tank, rng, whole)
        whole = stable_sort(tank, whole)
        slab = [stable_sort(tank, a) for a in slab]
        # every slab's owned layers and the ghost layer next to it are the
        # whole tank's, in the same order
        for r in range(nslabs):
            for z0, z1 in ((zb[r], zb[r + 1]), (zb[r] - 1, zb[r]), (zb[r + 1], zb[r + 1] + 1)):
                if z0 < 0 or z1 > NZ or z0 >= z1:
                    continue
                assert layer_slice(tank, slab[r], z0, z1) == layer_slice(tank, whole, z0, z1), (step, r, z0)
        # ---- splits of owned particles (children after the sorted count, in
        # slab order) and deaths
        whole_children = []
        children = [[] for _ in range(nslabs)]
        for r in range(nslabs):
            for i in layer_slice(tank, slab[r], zb[r], zb[r + 1]):
                u = rng.random()
                if u < 0.01:
                    j = tank.next_id
                    tank.next_id += 1
                    tank.z[j] = tank.z[i]
                    tank.c[j] = int(rng.integers(0, NXY))
                    children[r].append(j)
                    whole_children.append(j)
                elif u < 0.015:
                    tank.dead.add(i)
        # the whole tank's children come in the slabs' order, as their ids do
        assert whole_children == sum(children, [])


def test_slabs_create_rejects_bad_arguments_without_a_device():
    """Argument checks come before any device call (no GPU needed)."""
    L = cabi.load()
    h = cabi.C.c_void_p()
    fl = cabi.py_fluid(cabi.FLUID_LN2)
    rc = L.cryo_slabs_create(cabi.C.byref(cabi.py_config(dx=0.004)), cabi.C.byref(fl), 0, None, cabi.C.byref(h))
    assert rc == cabi.CRYO_EINVAL and not h.value
    assert b"slab" in L.cryo_slabs_last_error(None)
    rc = L.cryo_slabs_create(cabi.C.byref(cabi.py_config(dx=-1.0)), cabi.C.byref(fl), 2, None, cabi.C.byref(h))
    assert rc == cabi.CRYO_EINVAL and not h.value


@pytest.mark.parametrize("seed", range(20))
def test_partition_properties_random(seed):
    """Random layer counts: cuts increase, every slab keeps min_layers, and
    each cut lies where the running count first passes its share (or at the
    nearest cut the thickness rule allows)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nz = int(rng.integers(6, 80))
    nslabs = int(rng.integers(1, max(2, nz // 3) + 1))
    min_layers = int(rng.integers(1, nz // nslabs + 1))
    counts = rng.integers(0, 1000, size=nz) * (rng.random(nz) < 0.8)
    zb = cabi.slab_partition(counts, nslabs, min_layers=min_layers)
    assert zb[0] == 0 and zb[-1] == nz
    assert np.all(np.diff(zb) >= min_layers)
    total = int(counts.sum())
    cum = np.concatenate([[0], np.cumsum(counts)])
    for r in range(1, nslabs):
        target = (total * r + nslabs // 2) // nslabs
        lo = zb[r - 1] + min_layers
        hi = nz - (nslabs - r) * min_layers
        assert lo <= zb[r] <= hi
        # greedy: stops at the first layer whose inclusion would pass the target
        if lo < zb[r] < hi:
            assert cum[zb[r]] <= target < cum[zb[r] + 1]
