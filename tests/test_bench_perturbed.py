"""The plain method's GPU workload (bench.py --workload perturbed): seed-perturbed copies of the generated liner, each
breach connection's compiled area scaled by 1 + 0.02 i / count for instance i >= 1 (the reference's --perturb,
apps/sinksim_cuda_run.cpp:126-135, and this build's sinksim_cuda_run --perturb), instance 0 the compiled model; and the
reference arm's sweep document, which sets exactly those areas."""
import sys
import types

import numpy as np

from _support import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402
from sinksim_b200.files import load_model


def _args(count):
    return types.SimpleNamespace(workload="perturbed", count=count)


def test_perturbed_instances_scale_every_breach_like_the_reference_tool():
    ship_p, sim_p = bench.model_paths("liner")
    _, sim = load_model(ship_p, sim_p)
    count = 264
    params = bench.instance_params(sim, count, 0, _args(count))
    names = list(sim["kindNames"])
    breach = [c for c in range(len(sim["kind"])) if names[int(sim["kind"][c])] == "breach"]
    assert len(breach) > 0
    assert params[0] == ({}, {})
    for i in (1, 2, 131, 263):
        area, enabled = params[i]
        assert enabled == {} and sorted(area) == breach
        for c in breach:
            assert area[c] == float(sim["area"][c]) * (1 + 0.02 * i / count)
    # a shard starting at instance 100 of the same 264 draws the same values
    part = bench.instance_params(sim, 10, 100, _args(10), total=count)
    assert part == params[100:110]


def test_perturbed_sweep_document_sets_the_batch_areas():
    ship_p, sim_p = bench.model_paths("liner")
    _, sim = load_model(ship_p, sim_p)
    count = 12
    doc = bench.workload_sweep(sim, count, 9360.0, _args(count))
    assert doc["tMax"] == 9360.0 and len(doc["instances"]) == count
    params = bench.instance_params(sim, count, 0, _args(count))
    for inst, (area, _) in zip(doc["instances"], params):
        got = {e["conn"]: e["area"] for e in inst["connections"] if "area" in e}
        assert got == area
    assert bench.workload_rule(None, _args(count)) is None
