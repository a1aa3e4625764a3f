"""bench.py's two arms build the same workload from one plain-data spec: this
library's arm through the CryoSPH module, the reference arm through the
reference's own lattice generator (oracle/_ref) without importing anything of
the package.  These CPU tests check that both give identical inputs (config
fields, fluid, every particle array, domain) and that the checkers' struct
layouts (oracle/ref_abi.py) equal the package's (cryo_cabi)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import cryo_cabi as cabi
import ref_abi
import refpy

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

needs_ref = pytest.mark.skipif(not refpy.ref_available(), reason="reference CPU build (oracle/_ref) not built")


def _layout(cls):
    return [(name, C.sizeof(typ), getattr(cls, name).offset) for name, typ in cls._fields_]


@pytest.mark.parametrize("ours,theirs", [(cabi.Config, ref_abi.Config), (cabi.Fluid, ref_abi.Fluid),
                                         (cabi.Diagnostics, ref_abi.Diagnostics),
                                         (cabi.HostParticles, ref_abi.HostParticles)])
def test_checker_struct_layouts_match_the_package(ours, theirs):
    assert C.sizeof(ours) == C.sizeof(theirs)
    assert _layout(ours) == _layout(theirs)


def test_checker_tables_match_the_package():
    assert ref_abi.FIELDS == cabi.FIELDS and ref_abi.PASSES == cabi.PASSES
    assert ref_abi.CONFIG_DEFAULTS == cabi.CONFIG_DEFAULTS
    for which in cabi.FLUID_PRESETS:
        a, b = cabi.py_fluid(which), ref_abi.fluid(which)
        assert bytes(a) == bytes(b), which
    assert bytes(cabi.py_config(dx=0.01, thermal=0)) == bytes(ref_abi.config(dx=0.01, thermal=0))


def _c_config(cs_cfg):
    kw = {}
    for name, _ in cabi.CONFIG_FIELDS:
        v = getattr(cs_cfg, name)
        kw[name] = tuple(v) if name == "gravity" else (int(v.value) if hasattr(v, "value") else
                                                      (int(v) if isinstance(v, bool) else v))
    return cabi.py_config(**kw)


@needs_ref
@pytest.mark.parametrize("name,dx", [("dam_break", 0.04), ("c1", 0.006)])
def test_both_arms_build_identical_inputs(name, dx):
    import bench
    import CryoSPH as cs
    label, cfg, fluid, p, lo, hi = bench.workload(name, cs, dx)
    rlabel, rcfg, rfluid, rp, rlo, rhi = bench.ref_workload(name, dx)
    assert label == rlabel
    assert bytes(_c_config(cfg)) == bytes(rcfg)
    f = cabi.Fluid()
    for k, _ in cabi.Fluid._fields_:
        setattr(f, k, getattr(fluid, k))
    assert bytes(f) == bytes(rfluid)
    assert np.array_equal(np.asarray(lo, np.float32), np.asarray(rlo, np.float32))
    assert np.array_equal(np.asarray(hi, np.float32), np.asarray(rhi, np.float32))
    pairs = {"position": "x", "mass": "m", "density": "rho", "temperature": "T", "phase": "phase",
             "normal": "nrm", "flags": "flags"}
    for ours, theirs in pairs.items():
        a = np.asarray(p[ours])
        b = np.asarray(rp[theirs])
        if a.dtype.kind == "f":
            a, b = a.astype(np.float32), b.astype(np.float32)
        assert np.array_equal(a, b), ours
    n_wall = int((p["phase"] == 2).sum())
    assert bench.config_block(label, len(p["phase"]), len(p["phase"]) - n_wall, n_wall, 1) == \
        bench.config_block(rlabel, len(rp["phase"]), len(rp["phase"]) - n_wall, n_wall, 1)
