"""A sweep split into contiguous shards (what each GPU of a multi-GPU run takes) and merged in instance order gives
the whole sweep's results value for value, and the reference's comparer agrees. Both shards run on one GPU here,
one after the other: the shards never interact."""
import json
import subprocess

import pytest

import sinksim_b200 as ssb
from _support import fixture, ref_tool, titanic
from sinksim_b200.shard import merge_results

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_two_shards_merge_to_the_whole_sweep(tmp_path, numerics):
    ship_p, sim_p = titanic()
    sweep = fixture("smoke.sweep.json")
    whole = str(tmp_path / "whole.json")
    ssb.run_sweep(ship_p, sim_p, sweep, numerics, whole)
    parts = []
    for k, (first, count) in enumerate([(0, 2), (2, -1)]):
        p = str(tmp_path / f"part{k}.json")
        steps, _ = ssb.run_sweep_range(ship_p, sim_p, sweep, first, count, numerics, p)
        assert steps > 0
        with open(p) as f:
            parts.append(json.load(f))
    assert [len(p["instances"]) for p in parts] == [2, 3]
    merged = str(tmp_path / "merged.json")
    with open(merged, "w") as f:
        json.dump(merge_results(parts), f)
    compared, differing, first_diff = ssb.compare_results(whole, merged)
    assert compared > 1000 and differing == 0, first_diff
    r = subprocess.run([ref_tool("sinksim_sweep"), "--compare", whole, merged], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "RESULT: IDENTICAL" in r.stdout, r.stdout


def test_range_outside_the_sweep_is_refused(tmp_path):
    ship_p, sim_p = titanic()
    sweep = fixture("smoke.sweep.json")
    with pytest.raises(RuntimeError, match="do not exist"):
        ssb.run_sweep_range(ship_p, sim_p, sweep, 4, 2, "portable", str(tmp_path / "x.json"))
