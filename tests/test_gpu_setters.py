"""The block area setter (ssb_batch_set_connection_areas): a batch whose areas come from one block call runs bit for
bit as the same batch set one connection at a time through the reference's per-value setter; a block call with a bad
connection or instance range raises and writes nothing."""
import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import load_model, titanic

pytestmark = pytest.mark.gpu

COUNT = 6


def _run(setup):
    b = ssb.Batch(*titanic(), count=COUNT, t_max=900.0, curve_every=60.0)
    try:
        setup(b)
        b.run()
        return ([b.state(i).tolist() for i in range(COUNT)], [b.summary(i) for i in range(COUNT)],
                [b.curve(i).tolist() for i in range(COUNT)])
    finally:
        b.close()


def test_block_area_setter_equals_single_setters():
    _, sim = load_model(*titanic())
    n = len(sim["area"])
    rng = np.random.default_rng(11)
    conns = [int(c) for c in rng.choice(n, 40, replace=False)]
    areas = np.asarray(sim["area"], dtype=np.float64)[conns][None, :] * rng.lognormal(0.0, 0.3, (4, 40))

    def single(b):
        for i in range(4):
            for j, c in enumerate(conns):
                b.set_connection_area(1 + i, c, areas[i, j])

    def block(b):
        b.set_connection_areas(1, conns, areas)
        with pytest.raises(ssb.SinksimError):  # a connection out of range: nothing is written
            b.set_connection_areas(1, conns[:-1] + [n], 3.0 * areas)
        with pytest.raises(ssb.SinksimError):  # instances 3 .. 6 of 6: nothing is written
            b.set_connection_areas(3, conns, np.ones((4, 40)))

    assert _run(single) == _run(block)


def test_claim_order_must_be_a_permutation():
    b = ssb.Batch(*titanic(), count=4, t_max=60.0)
    try:
        for bad in ([0, 1, 2], [0, 1, 1, 3], [0, 1, 2, 4], [-1, 0, 1, 2]):
            with pytest.raises(ssb.SinksimError):
                b.set_claim_order(bad)
        b.set_claim_order([3, 2, 1, 0])
        b.run()
        assert all(b.summary(i)["steps"] == 240 for i in range(4))
        with pytest.raises(ssb.SinksimError):  # after the run
            b.set_claim_order([0, 1, 2, 3])
    finally:
        b.close()
