"""The drop-in tools' command lines on the CPU: usage errors exit 2 as the reference tools' do
(apps/cli.hpp:28-31, apps/sinksim_sweep.cpp:21-31 of the reference), numerics the GPU does not compute are refused
rather than replaced, and `sinksim_sweep --compare` (which needs no device) prints RESULT: IDENTICAL|DIFFERENT with
exit 0 / 1 on batch-results files."""
import json
import os
import subprocess

import pytest

from _support import ROOT

BIN = os.path.join(ROOT, "sinksim_b200", "bin")


def tool(name, *args):
    return subprocess.run([os.path.join(BIN, name), *args], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args", [[], ["ship.json"], ["a", "b"], ["a", "b", "c"], ["a", "b", "c", "--numerics", "oracle"],
                                  ["a", "b", "c", "--numerics", "std"], ["a", "b", "c", "--numerics", "nope"], ["--compare"],
                                  ["--compare", "a.json"], ["a", "b", "c", "--results"]])
def test_sinksim_sweep_usage_errors_exit_2(args):
    r = tool("sinksim_sweep", *args)
    assert r.returncode == 2, (args, r.stdout, r.stderr)


def test_sinksim_sweep_names_the_missing_numerics():
    r = tool("sinksim_sweep", "a", "b", "c")
    assert "--numerics" in r.stderr and "oracle" in r.stderr


@pytest.mark.parametrize("args", [[], ["ship.json"], ["a", "b", "--precision", "single"], ["a", "b", "--numerics", "oracle"],
                                  ["a", "b", "--count"], ["a", "b", "--count", "x"]])
def test_sinksim_cuda_run_usage_errors_exit_2(args):
    r = tool("sinksim_cuda_run", *args)
    assert r.returncode == 2, (args, r.stdout, r.stderr)


def test_missing_files_fail_with_exit_1(tmp_path):
    r = tool("sinksim_sweep", str(tmp_path / "no.ship.json"), str(tmp_path / "no.sim.json"), str(tmp_path / "no.sweep.json"), "--numerics", "portable")
    assert r.returncode == 1 and r.stderr.startswith("sinksim_sweep:")


def _results(trim_last):
    inst = {"id": "a", "foundered": False, "founderT": -1, "tEnd": 10, "steps": 40,
            "final": {"trimDeg": 0.5, "listDeg": 0, "waterT": 1, "draftF": 2, "draftA": 3, "inflowTpm": 0}, "events": [],
            "curve": {"t": [0, 5, 10], "trim": [0, 0.25, trim_last], "list": [0, 0, 0], "water": [0, 0.5, 1], "inflow": [0, 0, 0],
                      "draftF": [2, 2, 2], "draftA": [3, 3, 3]}}
    return {"format": "sinksim.batch-results", "formatVersion": 1, "ship": "s", "sim": "m", "numerics": "portable", "engine": "e",
            "tMax": 10, "every": 5, "instances": [inst]}


def test_compare_identical_and_different(tmp_path):
    a, b = tmp_path / "a.json", tmp_path / "b.json"
    a.write_text(json.dumps(_results(0.5)))
    b.write_text(json.dumps(_results(0.5000000000000001)))
    same = tool("sinksim_sweep", "--compare", str(a), str(a))
    assert same.returncode == 0 and "RESULT: IDENTICAL" in same.stdout
    diff = tool("sinksim_sweep", "--compare", str(a), str(b))
    assert diff.returncode == 1 and "RESULT: DIFFERENT" in diff.stdout and "curve[2] trim" in diff.stdout
