"""The C-ABI library without a GPU: it loads, exports every entry point that
include/cryosph_b200.h declares, and its host-side functions (defaults,
presets, Clausius-Clapeyron, manoeuvre interpolation, argument validation)
behave like the reference's."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import cryo_cabi as cabi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "cryosph_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cryo_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = cabi.load()
    names = declared_functions()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.cryo_abi_version() == 1


def test_config_defaults_match_solverconfig():
    a = cabi.config_default()
    b = cabi.py_config()
    for name, _ in cabi.CONFIG_FIELDS:
        va, vb = getattr(a, name), getattr(b, name)
        if isinstance(va, C.Array):
            assert list(va) == list(vb), name
        else:
            assert va == pytest.approx(vb, rel=0, abs=0), name


@pytest.mark.parametrize("which", range(6))
def test_fluid_presets(which):
    f = cabi.fluid_preset(which)
    g = cabi.py_fluid(which)
    for name, _ in cabi.Fluid._fields_:
        assert np.float32(getattr(f, name)) == np.float32(getattr(g, name)), name


def test_clausius_clapeyron_roundtrip():
    L = cabi.load()
    ln2 = cabi.fluid_preset(cabi.FLUID_LN2)
    assert L.cryo_saturation_temperature(C.byref(ln2), ln2.p_sat) == pytest.approx(ln2.T_sat, rel=1e-6)
    p2 = L.cryo_saturation_pressure(C.byref(ln2), ln2.T_sat + 2.0)
    assert p2 > ln2.p_sat
    assert L.cryo_saturation_temperature(C.byref(ln2), p2) == pytest.approx(ln2.T_sat + 2.0, rel=1e-5)


def test_create_rejects_bad_config_without_touching_the_device():
    L = cabi.load()
    h = C.c_void_p()
    fl = cabi.fluid_preset(cabi.FLUID_LN2)
    rc = L.cryo_create(C.byref(cabi.config_default(dx=0.0)), C.byref(fl), 0, C.byref(h))
    assert rc == cabi.CRYO_EINVAL and not h.value
    assert b"dx" in L.cryo_last_error(None)
    rc = L.cryo_create(C.byref(cabi.config_default(contact_angle_deg=200.0)), C.byref(fl), 0, C.byref(h))
    assert rc == cabi.CRYO_EINVAL and b"contact angle" in L.cryo_last_error(None)


def test_maneuver_interpolation():
    """test_maneuver.cpp:34-56 through cryo_maneuver_evaluate."""
    L = cabi.load()
    t = (C.c_double * 3)(0.0, 1.0, 3.0)
    acc = (C.c_float * 9)(0, 0, 0, 2, 0, 0, 2, 0, 0)
    om = (C.c_float * 9)(0, 0, 0, 0, 0, 1, 0, 0, 0)
    a, w, wd = (C.c_float * 3)(), (C.c_float * 3)(), (C.c_float * 3)()

    def ev(tq):
        assert L.cryo_maneuver_evaluate(3, t, acc, om, tq, a, w, wd) == 0
        return list(a), list(w), list(wd)

    a0, w0, wd0 = ev(0.5)
    assert a0[0] == pytest.approx(1.0) and w0[2] == pytest.approx(0.5) and wd0[2] == pytest.approx(1.0)
    a1, w1, wd1 = ev(2.0)
    assert w1[2] == pytest.approx(0.5) and wd1[2] == pytest.approx(-0.5)
    a2, w2, wd2 = ev(10.0)
    assert a2[0] == pytest.approx(2.0) and wd2[2] == 0.0
    assert L.cryo_maneuver_evaluate(0, t, acc, om, 0.0, a, w, wd) == cabi.CRYO_EINVAL


def test_host_structs_match_header_sizes():
    # the C structs are plain floats/ints: sizes follow the field lists
    assert C.sizeof(cabi.Fluid) == 13 * 4
    assert C.sizeof(cabi.Config) == (len(cabi.CONFIG_FIELDS) + 2) * 4
