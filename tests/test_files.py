"""Refusing bad input files on the host, before any device work: the checks of the reference's loaders
(engine/src/compiled.cpp:82-279, engine/src/sweep.cpp:25-70) with the engine's error codes.

A compiled file whose values were changed after it was written no longer matches the hashes it states (one changed
value is enough), a file of another format or version is not read, a sim compiled for another ship is refused, and a
sweep naming a connection kind the sim does not have is refused. Each returns SSB_ERUNTIME (-2) with the reason.
"""
import json

import pytest

import sinksim_b200 as ssb
from _support import titanic


def _doc(path):
    with open(path) as f:
        return json.load(f)


def _write(tmp_path, name, doc):
    p = tmp_path / name
    p.write_text(json.dumps(doc))
    return str(p)


def _refused(ship, sim, sweep=None):
    with pytest.raises(ssb.SinksimError) as e:
        ssb.check_model(ship, sim, sweep)
    assert e.value.code == -2
    return str(e.value)


def test_the_pristine_files_pass():
    ship, sim = titanic()
    ssb.check_model(ship, sim)


def test_one_changed_ship_value_is_a_hash_mismatch(tmp_path):
    ship, sim = titanic()
    d = _doc(ship)
    d["columns"]["x"][17] += 1e-9
    msg = _refused(_write(tmp_path, "ship.json", d), sim)
    assert "hash mismatch on columns.x" in msg


def test_one_changed_sim_value_is_a_hash_mismatch(tmp_path):
    ship, sim = titanic()
    d = _doc(sim)
    d["connections"]["area"][3] *= 1.5
    msg = _refused(ship, _write(tmp_path, "sim.json", d))
    assert "hash mismatch on connections.area" in msg


def test_a_stated_hash_that_was_edited_is_a_mismatch(tmp_path):
    ship, sim = titanic()
    d = _doc(ship)
    d["hash"]["all"] = "0" * 16
    assert "hash mismatch" in _refused(_write(tmp_path, "ship.json", d), sim)


def test_other_formats_and_versions_are_not_read(tmp_path):
    ship, sim = titanic()
    d = _doc(ship)
    d["formatVersion"] = 2
    assert "formatVersion 2" in _refused(_write(tmp_path, "v2.json", d), sim)
    d = _doc(ship)
    d["format"] = "sinksim.compiled-sim"
    assert "sinksim.compiled-ship" in _refused(_write(tmp_path, "fmt.json", d), sim)


def test_a_length_that_does_not_match_the_count_is_refused(tmp_path):
    ship, sim = titanic()
    d = _doc(ship)
    d["columns"]["zhi"] = d["columns"]["zhi"][:-1]
    assert "columns.zhi" in _refused(_write(tmp_path, "short.json", d), sim)


def test_a_sim_for_another_ship_is_refused(tmp_path):
    from sinksim_b200 import hullgen

    ship, sim = titanic()
    liner_ship, liner_sim = hullgen.write(str(tmp_path))
    assert "belongs to ship" in _refused(liner_ship, sim)


def test_a_sweep_with_an_unknown_kind_is_refused(tmp_path):
    ship, sim = titanic()
    sweep = {"format": "sinksim.sweep", "formatVersion": 1, "instances": [{"id": "x", "scale": {"portholes": 2.0}}]}
    assert "portholes" in _refused(ship, sim, _write(tmp_path, "sweep.json", sweep))
    sweep["formatVersion"] = 3
    assert "formatVersion" in _refused(ship, sim, _write(tmp_path, "sweep3.json", sweep))
    ok = {"format": "sinksim.sweep", "formatVersion": 1, "instances": [{"id": "x", "scale": {"breach": 2.0}}]}
    ssb.check_model(ship, sim, _write(tmp_path, "ok.json", ok))
