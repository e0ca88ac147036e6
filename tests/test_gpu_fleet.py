"""A fleet: instances of several generated hulls stepped in the same launches. Every instance's results equal those
of a batch of its own model alone (state, summary, curve, events; bit for bit, both numerics), and one instance of
each hull equals the reference CPU engine."""
import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import RefSim, load_model
from sinksim_b200 import hullgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hulls(tmp_path_factory):
    d = tmp_path_factory.mktemp("fleet")
    specs = hullgen.fleet_specs(3, seed=11, columns=(1000, 3000))
    return [hullgen.write(str(d), spec=sp, seed=20 + i, ship_id=f"hull{i}") for i, sp in enumerate(specs)]


def _settings(sim, k):
    """Instance k's breach scale (areas of the breach connections)."""
    kinds = list(sim["kindNames"])
    br = np.nonzero(np.asarray(sim["kind"]) == kinds.index("breach"))[0]
    return {int(c): float(sim["area"][c]) * (0.6 + 0.2 * k) for c in br}


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_fleet_equals_each_model_alone(hulls, numerics):
    t_max, every = 2400.0, 120.0
    sims = [load_model(*h)[1] for h in hulls]
    instance_model = [0, 1, 2, 2, 0, 1, 0, 2, 1]
    fleet = ssb.Batch.fleet(hulls, instance_model, numerics=numerics, t_max=t_max, curve_every=every)
    for i, m in enumerate(instance_model):
        for c, a in _settings(sims[m], i).items():
            fleet.set_connection_area(i, c, a)
    fleet.run()
    for m, (ship_p, sim_p) in enumerate(hulls):
        mine = [i for i, mm in enumerate(instance_model) if mm == m]
        with ssb.Batch(ship_p, sim_p, count=len(mine), numerics=numerics, t_max=t_max, curve_every=every) as alone:
            for j, i in enumerate(mine):
                for c, a in _settings(sims[m], i).items():
                    alone.set_connection_area(j, c, a)
            alone.run()
            for j, i in enumerate(mine):
                assert fleet.instance_shape(i)[0] == m
                np.testing.assert_array_equal(fleet.state(i), alone.state(j), err_msg=f"model {m} instance {i}")
                a, b = fleet.summary(i), alone.summary(j)
                assert (a["steps"], a["foundered"], a["founder_t"], a["t_end"]) == (b["steps"], b["foundered"], b["founder_t"], b["t_end"])
                np.testing.assert_array_equal(fleet.curve(i), alone.curve(j))
                assert fleet.events(i) == alone.events(j)
    fleet.close()


def test_fleet_instances_equal_the_reference_engine(hulls):
    t_max = 1200.0
    sims = [load_model(*h)[1] for h in hulls]
    instance_model = [2, 0, 1]
    fleet = ssb.Batch.fleet(hulls, instance_model, numerics="portable", t_max=t_max)
    for i, m in enumerate(instance_model):
        for c, a in _settings(sims[m], i).items():
            fleet.set_connection_area(i, c, a)
    fleet.run()
    for i, m in enumerate(instance_model):
        ref = RefSim(*hulls[m], "portable")
        for c, a in _settings(sims[m], i).items():
            ref.set_connection(c, area=a)
        ref.step(fleet.summary(i)["steps"])
        np.testing.assert_array_equal(fleet.state(i), ref.record(), err_msg=f"instance {i}")
    fleet.close()
