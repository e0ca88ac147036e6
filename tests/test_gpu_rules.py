"""Retiring instances early, on a B200, against the reference CPU engine.

  * The batching workloads' sink/settle rule: the reference runs it through Simulation::run's onStep hook
    (engine/src/simulation.cpp:183; oracle/ref_harness.cpp); the GPU evaluates it in the kernel after every step.
    Steps, end time, founder flag and time, the rule that fired, the readout curve and the final state must match.
  * The reference's own "stopWhenStable" calm rule (simulation.cpp:179-182), which its GPU runner refused: a sweep
    with stopWhenStable run by the drop-in must equal the reference sweep tool's results value for value.
"""
import json
import subprocess

import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import RefSim, load_model, ref_tool, titanic
from sinksim_b200.workloads import batch_uneven, deck_edge_rule

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_retire_rule_matches_reference_onstep(numerics):
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    rule = deck_edge_rule(ship)
    # instances of the uneven-length batch: 1, 7 and 10 end by the sink rule, 0, 2 and 13 by the settle rule
    picks = [0, 1, 2, 7, 10, 13]
    params = batch_uneven(sim, max(picks) + 1)
    count = len(picks)
    t_max = 5 * 3600.0
    b = ssb.Batch(ship_p, sim_p, count=count, numerics=numerics, t_max=t_max, curve_every=60.0, rule=rule)
    for i, k in enumerate(picks):
        area, enabled = params[k]
        for c, a in area.items():
            b.set_connection_area(i, c, a)
        for c, e in enabled.items():
            b.set_connection_enabled(i, c, e)
    b.run()
    rule_vec = [rule[k] for k in ("pitch", "x", "y", "z", "wth", "settle")]
    why = {0: ("foundered", "tmax"), 1: ("sink-rule",), 2: ("settle-rule",)}
    seen = set()
    for i, k in enumerate(picks):
        ref = RefSim(ship_p, sim_p, numerics)
        area, enabled = params[k]
        for c, a in area.items():
            ref.set_connection(c, area=a)
        for c, e in enabled.items():
            ref.set_connection(c, enabled=e)
        summary, curve = ref.run(t_max, 60.0, rule=rule_vec)
        s = b.summary(i)
        assert s["steps"] == summary["steps"], f"instance {k}"
        assert s["t_end"] == summary["tEnd"]
        assert s["foundered"] == summary["foundered"] and s["founder_t"] == summary["founderT"]
        assert s["stop"] in why[summary["retired"]], (k, s["stop"], summary["retired"])
        seen.add(summary["retired"])
        np.testing.assert_array_equal(b.curve(i), curve, err_msg=f"instance {k} curve")
        np.testing.assert_array_equal(b.state(i), ref.record(), err_msg=f"instance {k} state")
    b.close()
    assert {1, 2} <= seen  # both rules were exercised


def test_stop_when_stable_sweep_equals_reference_sweep(tmp_path):
    ship_p, sim_p = titanic()
    sweep = {"format": "sinksim.sweep", "formatVersion": 1, "ship": "titanic64", "sim": "titanic", "tMax": 5 * 3600, "every": 30,
             "stopWhenStable": True,
             "instances": [{"id": f"breach-{f}", "scale": {"breach": f}} for f in (0.0, 0.001, 0.005, 0.3, 1.0)] +
                          [{"id": "breaches-closed", "connections": [{"kind": "breach", "enabled": False}]}]}
    sp = tmp_path / "stable.sweep.json"
    sp.write_text(json.dumps(sweep))
    cpu, gpu = str(tmp_path / "cpu.json"), str(tmp_path / "gpu.json")
    r = subprocess.run([ref_tool("sinksim_sweep"), ship_p, sim_p, str(sp), "--numerics", "portable", "--results", cpu],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    ssb.run_sweep(ship_p, sim_p, str(sp), "portable", gpu)
    compared, differing, first = ssb.compare_results(cpu, gpu)
    assert differing == 0, first
    res = json.load(open(gpu))
    # the calm rule must have ended some runs early (neither founder nor tMax)
    assert any((not x["foundered"]) and x["tEnd"] < 5 * 3600 for x in res["instances"])
