"""The launch-shape autotuner on a small uneven batch: it times every candidate, returns the fastest, and the tuned
batch's results equal the default shape's bit for bit."""
import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import load_model, titanic
from sinksim_b200.autotune import tune
from sinksim_b200.workloads import batch_uneven, deck_edge_rule

pytestmark = pytest.mark.gpu


def test_tuned_shape_is_timed_and_changes_no_result():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    rule = deck_edge_rule(ship)
    params = batch_uneven(sim, 96)

    def make(**shape):
        b = ssb.Batch(ship_p, sim_p, count=96, numerics="portable", t_max=1800.0, rule=rule, **shape)
        for i, (area, en) in enumerate(params):
            for c, a in area.items():
                b.set_connection_area(i, c, a)
            for c, e in en.items():
                b.set_connection_enabled(i, c, e)
        return b

    candidates = ({}, {"team_warps": 1}, {"team_warps": 8, "tail_team_warps": 0})
    best, table = tune(make, candidates)
    assert len(table) == 3 and all(ms > 0 for _, ms, _ in table)
    assert best == min(table, key=lambda r: r[1])[0]
    a, b = make(), make(**best)
    a.run()
    b.run()
    assert a.total_steps() == b.total_steps() == table[0][2]
    for i in range(96):
        np.testing.assert_array_equal(a.state(i), b.state(i))
    a.close()
    b.close()
