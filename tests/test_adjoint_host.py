"""Host-side pieces of the differentiated window (no GPU): the knot schedule
of cryo_adjoint.slosh_window gives every step exactly one knot."""
import numpy as np

import cryo_adjoint as ca

DT = 1e-3


def test_knot_schedule_gives_each_step_one_knot():
    for steps, k in ((8, 4), (400, 16), (10, 3), (5, 5)):
        times, seg = ca.knot_schedule(0.125, DT, steps, k)
        assert np.all(np.diff(times) > 0)
        prof = ca._maneuver(times, np.arange(3 * k, dtype=np.float64).reshape(k, 3))
        for n in range(steps):
            a = prof.evaluate(0.125 + (n + 1) * DT)[0]
            assert abs(a[0] - 3 * seg[n]) <= 1e-5 * max(1.0, 3 * seg[n])
        assert np.all(np.diff(seg) >= 0) and seg[0] == 0 and seg[-1] == k - 1
        assert len(np.unique(seg)) == k


def test_knot_schedule_rejects_more_knots_than_steps():
    import pytest
    with pytest.raises(ValueError):
        ca.knot_schedule(0.0, DT, 3, 4)
