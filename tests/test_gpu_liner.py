"""The generated benchmark liner on the GPU: the trace of a batch instance passes the reference's own checker at
tolerance 0 (the reference CPU engine re-run window by window), and a perturbed sweep of the liner gives the reference
CPU sweep's results value for value, in both numerics."""
import json
import subprocess

import pytest

import sinksim_b200 as ssb
from _support import ref_tool
from sinksim_b200 import hullgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def liner(tmp_path_factory):
    return hullgen.write(str(tmp_path_factory.mktemp("liner")))


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_liner_trace_passes_the_reference_checker(liner, tmp_path, numerics):
    ship_p, sim_p = liner
    path = str(tmp_path / "gpu.trace.json")
    with ssb.Batch(ship_p, sim_p, count=4, numerics=numerics, traced_instances=1, dense_steps=400, sample_every=60.0) as b:
        b.run()
        s = b.summary(0)
        assert s["foundered"] and 1200 < s["founder_t"] < 18000
        b.save_trace(0, path)
    r = subprocess.run([ref_tool("sinksim_check"), ship_p, sim_p, path, "--numerics", numerics, "--tol-step", "0", "--tol-window", "0", "--quiet"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "RESULT: PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_liner_sweep_equals_reference_cpu_sweep(liner, tmp_path, numerics):
    ship_p, sim_p = liner
    instances = [{"id": "base"}]
    for i in range(1, 8):
        inst = {"id": f"p{i}", "scale": {"breach": 0.5 + 0.25 * i, "down": 1.0 + 0.1 * i}}
        if i % 2:
            inst["connections"] = [{"conn": 1 + 8 * i, "enabled": True}]     # open a door
        instances.append(inst)
    sweep = {"format": "sinksim.sweep", "formatVersion": 1, "ship": "liner269.ship.json", "sim": "liner269.sim.json", "tMax": 9000,
             "every": 120, "stopWhenStable": False, "instances": instances}
    sw = str(tmp_path / "liner.sweep.json")
    with open(sw, "w") as f:
        json.dump(sweep, f)
    cpu, gpu = str(tmp_path / "cpu.json"), str(tmp_path / "gpu.json")
    r = subprocess.run([ref_tool("sinksim_sweep"), ship_p, sim_p, sw, "--numerics", numerics, "--results", cpu], capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    ssb.run_sweep(ship_p, sim_p, sw, numerics, gpu)
    compared, differing, first = ssb.compare_results(cpu, gpu)
    assert compared > 1000 and differing == 0, first
