"""The run's health report (ssb_batch_health): a condition set on the host (a NaN in one instance's restored volume)
surfaces as the non-finite flag after the run, the other instances keep their bits, and a clean run reports nothing.
No GPU fault is involved: the kernel records the condition in its error word and the host reads it back."""
import math

import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import Oracle, load_model, titanic

pytestmark = pytest.mark.gpu


def test_a_nan_state_surfaces_as_the_non_finite_flag():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    nn = len(ship["mu"])
    with ssb.Batch(ship_p, sim_p, count=3, numerics="portable", t_max=120.0) as b:
        b.run()
        assert b.health() == 0
        clean = [b.state(i) for i in range(3)]
    with ssb.Batch(ship_p, sim_p, count=3, numerics="portable", t_max=120.0) as b:
        o = Oracle(ship, sim, False)
        rec = o.record()
        rec[10 + nn // 2] = math.nan  # one node's volume
        b.restore(1, rec)
        b.run()
        assert b.health() & ssb.HEALTH_NON_FINITE
        assert not np.isfinite(b.state(1)[1])
        for i in (0, 2):
            np.testing.assert_array_equal(b.state(i), clean[i])
