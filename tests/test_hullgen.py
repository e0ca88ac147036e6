"""The synthetic hull compiler: the benchmark liner has the stated shape, is the same for the same seed, loads in the
reference's own tools (which verify every hash), and the C restatement steps it bit for bit like the reference engine
(single-node groups, four decks of segments per column: shapes the titanic model does not have)."""
import json
import subprocess

import numpy as np
import pytest

from _support import Oracle, RefSim, load_model, ref_tool
from sinksim_b200 import hullgen


@pytest.fixture(scope="module")
def liner(tmp_path_factory):
    d = tmp_path_factory.mktemp("liner")
    return hullgen.write(str(d))


def test_liner_shape(liner):
    ship_p, sim_p = liner
    with open(ship_p) as f:
        ship = json.load(f)
    with open(sim_p) as f:
        sim = json.load(f)
    assert ship["columns"]["n"] == 152 * 29 == 4408
    assert ship["nodes"]["n"] == 64 and sim["groups"]["n"] == 64
    assert sim["connections"]["n"] == 290
    kinds = sim["connections"]["kindNames"]
    k = np.array(sim["connections"]["kind"])
    breach = (k == kinds.index("breach")) & (np.array(sim["connections"]["en"]) == 1)
    assert breach.sum() == 6                                   # six open breaches, and two closed ones aft of them
    assert (k == kinds.index("breach")).sum() == 8
    assert np.isclose(np.array(sim["connections"]["area"])[breach].sum(), 1.2)
    doors = np.array(sim["connections"]["area"])[k == kinds.index("door")]
    assert doors.min() >= 1.0 and doors.max() <= 3.0
    assert sim["shipHash"] == ship["hash"]["all"]
    assert abs(ship["hydrostatics"]["KB"] + ship["hydrostatics"]["BM"] - sim["body"]["KG"] - 0.8) < 1e-9


def test_same_seed_same_files(tmp_path):
    a = hullgen.generate(seed=7)
    b = hullgen.generate(seed=7)
    c = hullgen.generate(seed=8)
    assert a[0]["hash"] == b[0]["hash"] and a[1]["hash"] == b[1]["hash"]
    assert a[0]["hash"]["all"] == c[0]["hash"]["all"]      # the hull does not depend on the seed
    assert a[1]["hash"]["all"] != c[1]["hash"]["all"]      # the connections do


def test_reference_tools_load_and_run_the_liner(liner, tmp_path):
    ship_p, sim_p = liner
    r = subprocess.run([ref_tool("sinksim_run"), ship_p, sim_p, "--numerics", "portable", "--tmax", "600"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.parametrize("mixed", [False, True])
def test_restatement_steps_the_liner_like_the_reference(liner, mixed):
    ship_p, sim_p = liner
    ship, sim = load_model(ship_p, sim_p)
    ref = RefSim(ship_p, sim_p, "portable32" if mixed else "portable")
    ora = Oracle(ship, sim, mixed=mixed)
    for c in (3, 17, 150):                       # open a few doors and widen a deck opening on both
        ref.set_connection(c, enabled=1)
        ora.set_connection(c, enabled=1)
    for chunk in (1, 99, 900, 3000):
        ref.step(chunk)
        ora.step(chunk)
        np.testing.assert_array_equal(ora.record(), ref.record())


def test_fleet_specs_cover_the_configured_ranges():
    specs = hullgen.fleet_specs(24, seed=5)
    for i, sp in enumerate(specs):
        ship, sim = hullgen.generate(sp, seed=i, ship_id=f"h{i}")
        cols, spaces = ship["columns"]["n"], ship["nodes"]["n"]
        assert 900 <= cols <= 21000, cols
        assert 16 <= spaces <= 256, spaces
        assert 3 <= sim["connections"]["n"] / spaces <= 5, sim["connections"]["n"] / spaces
        assert 100 <= sp.L <= 300
