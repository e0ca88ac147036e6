"""The C restatement of the step (oracle/sinksim_oracle.c) is pinned, before anything is checked against it:
  * to the reference's golden traces of titanic64 (tolerance 0, as the reference's own CTest golden_portable and
    golden_portable32 tests, tests/CMakeLists.txt:19-28): the initial record, one step from each dense record, and
    the whole run from the initial state through every sampled record;
  * to the reference CPU engine itself (oracle/_ref, built from the reference sources), step for step with
    connection changes, flows and events included.
"""
import os

import numpy as np
import pytest

from _support import GOLDEN, Oracle, RefSim, load_model, read_json, titanic, trace_records


@pytest.fixture(scope="module")
def model():
    ship_p, sim_p = titanic()
    return ship_p, sim_p, *load_model(ship_p, sim_p)


@pytest.mark.parametrize("tag,mixed", [("portable", False), ("portable32", True)])
def test_dense_steps_match_golden(model, tag, mixed):
    _, _, ship, sim = model
    g = read_json(os.path.join(GOLDEN, f"titanic.{tag}.golden.json.gz"))
    dense = trace_records(g, "dense")
    o = Oracle(ship, sim, mixed)
    assert np.array_equal(o.record(), dense[0])
    for i in range(len(dense) - 1):
        o.restore(dense[i])
        o.step(1)
        np.testing.assert_array_equal(o.record(), dense[i + 1], err_msg=f"step {i + 1}")


@pytest.mark.parametrize("tag,mixed", [("portable", False), ("portable32", True)])
def test_end_to_end_matches_golden_samples(model, tag, mixed):
    _, _, ship, sim = model
    g = read_json(os.path.join(GOLDEN, f"titanic.{tag}.golden.json.gz"))
    samples = trace_records(g, "samples")
    o = Oracle(ship, sim, mixed)
    for i in range(len(samples) - 1):
        o.step(int(round((samples[i + 1, 0] - samples[i, 0]) / sim["dt"])))
        np.testing.assert_array_equal(o.record(), samples[i + 1], err_msg=f"sample {i + 1}")
    # run on to the founder and compare the event log (ids and times) with the golden's
    while not o.foundered()[0] and o.record()[0] < 5 * 3600:
        o.step(1)
    assert o.foundered() == (g["foundered"], g["founderT"])
    ev = o.events()
    assert len(ev) == len(g["events"])
    names = {0: sim["monitorId"], 1: sim["markId"]}
    for (t, i, kind), e in zip(ev, g["events"]):
        assert t == e["t"]
        assert (names[kind][i] if kind in names else "founder") == e["id"]


def test_work_counts_titanic64(model):
    """The per-step work the roofline figures use: clipped columns, node passes, segment visits, weir pows."""
    _, _, ship, sim = model
    o = Oracle(ship, sim, False)
    c0 = o.counters()
    o.step(2000)
    c = {k: v - c0[k] for k, v in o.counters().items()}
    assert c["columns"] == 2000 * len(ship["x"])
    assert 60 < c["passes"] / 2000 < 80
    assert 8000 < c["segVisits"] / 2000 < 11000


@pytest.mark.parametrize("numerics,mixed", [("portable", False), ("portable32", True)])
def test_matches_reference_engine_with_connection_changes(model, numerics, mixed):
    ship_p, sim_p, ship, sim = model
    ref = RefSim(ship_p, sim_p, numerics)
    o = Oracle(ship, sim, mixed)
    rng = np.random.default_rng(7)
    kinds = sim["kind"]
    for c in np.nonzero(kinds == kinds[-1])[0]:
        a = sim["area"][c] * 1.37
        ref.set_connection(int(c), area=a)
        o.set_connection(int(c), area=a)
    for c in rng.choice(len(sim["ca"]), 12, replace=False):
        t_on = float(rng.uniform(0, 600))
        ref.set_connection(int(c), enabled=1, tOn=t_on)
        o.set_connection(int(c), enabled=1, tOn=t_on)
    for k in range(40):
        ref.step(50)
        o.step(50)
        np.testing.assert_array_equal(o.record(), ref.record(), err_msg=f"after {50 * (k + 1)} steps")
    np.testing.assert_array_equal(o.readouts(), ref.readouts())
    assert o.events() == ref.events()
