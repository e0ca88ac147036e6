"""Parity of the CUDA batch engine with the reference, on a B200, through the C ABI.

  * titanic64 in portable and portable32: the trace of instance 0 of a batch of 8 reproduces the reference's golden
    trace at tolerance 0 (every committed dense record, every sampled record, the events and the founder time), and
    the reference's own checker (oracle/_ref/sinksim_check, built from the reference sources) passes it at
    --tol-step 0 --tol-window 0: the reference's cuda_matches_portable[32] acceptance tests (tests/CMakeLists.txt:40-57).
  * the smoke sweep: the GPU's batch-results equal the reference CPU engine's (oracle/_ref/sinksim_sweep) value for
    value, as the reference's sweep_gpu_matches_cpu test requires (tests/CMakeLists.txt:59-65), in both numerics.
  * perturbed batches: every instance's final state equals the C restatement (oracle/) stepped from the same inputs.
  * launch shape: bounded launches and other simulations-per-block give the same bits.
"""
import os
import subprocess

import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import GOLDEN, Oracle, fixture, load_model, read_json, ref_tool, titanic, trace_records

pytestmark = pytest.mark.gpu

NUMERICS = [("portable", False), ("portable32", True)]


@pytest.fixture(scope="module")
def model():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    return ship_p, sim_p, ship, sim


@pytest.mark.parametrize("numerics,mixed", NUMERICS)
def test_trace_matches_golden_and_reference_checker(model, tmp_path, numerics, mixed):
    ship_p, sim_p, ship, sim = model
    g = read_json(os.path.join(GOLDEN, f"titanic.{numerics}.golden.json.gz"))
    with ssb.Batch(ship_p, sim_p, count=8, numerics=numerics, traced_instances=1, dense_steps=400, sample_every=60.0) as b:
        b.run()
        path = str(tmp_path / f"cuda.{numerics}.trace.json")
        b.save_trace(0, path)
        s = b.summary(0)
        assert s["foundered"] == g["foundered"] and s["founder_t"] == g["founderT"]
        assert s["steps"] == g["steps"]
        ev = b.events(0)
        assert [e[0] for e in ev] == [e["t"] for e in g["events"]]
    tr = read_json(path)
    dense, gd = trace_records(tr, "dense"), trace_records(g, "dense")
    assert tr["dense"]["n"] == 401
    np.testing.assert_array_equal(dense[: len(gd)], gd)
    samples, gs = trace_records(tr, "samples"), trace_records(g, "samples")
    assert samples.shape == gs.shape
    np.testing.assert_array_equal(samples, gs)
    r = subprocess.run([ref_tool("sinksim_check"), ship_p, sim_p, path, "--numerics", numerics, "--tol-step", "0", "--tol-window", "0", "--quiet"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "RESULT: PASS" in r.stdout, r.stdout + r.stderr


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_smoke_sweep_equals_reference_cpu_sweep(model, tmp_path, numerics):
    ship_p, sim_p, _, _ = model
    sweep = fixture("smoke.sweep.json")
    cpu = str(tmp_path / "cpu.json")
    gpu = str(tmp_path / "gpu.json")
    r = subprocess.run([ref_tool("sinksim_sweep"), ship_p, sim_p, sweep, "--numerics", numerics, "--results", cpu],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    steps, secs = ssb.run_sweep(ship_p, sim_p, sweep, numerics, gpu)
    assert steps > 0
    compared, differing, first = ssb.compare_results(cpu, gpu)
    assert compared > 1000 and differing == 0, first
    # and the reference's own comparer agrees
    r = subprocess.run([ref_tool("sinksim_sweep"), "--compare", cpu, gpu], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "RESULT: IDENTICAL" in r.stdout, r.stdout


def _perturbed_batch(ship_p, sim_p, sim, count, numerics, t_max, **kw):
    kinds = sim["kindNames"]
    breach = kinds.index("breach") if "breach" in kinds else -1
    b = ssb.Batch(ship_p, sim_p, count=count, numerics=numerics, t_max=t_max, **kw)
    areas = {}
    for i in range(1, count):
        scale = 1 + 0.02 * i / count
        for c in np.nonzero(sim["kind"] == breach)[0]:
            a = sim["area"][c] * scale
            b.set_connection_area(i, int(c), a)
            areas[(i, int(c))] = a
    return b, areas


@pytest.mark.parametrize("numerics,mixed", NUMERICS)
def test_perturbed_batch_equals_oracle(model, numerics, mixed):
    ship_p, sim_p, ship, sim = model
    count, t_max = 12, 2400.0
    b, areas = _perturbed_batch(ship_p, sim_p, sim, count, numerics, t_max, curve_every=30.0)
    b.run()
    for i in range(count):
        o = Oracle(ship, sim, mixed)
        for (j, c), a in areas.items():
            if j == i:
                o.set_connection(c, area=a)
        curve = []
        nxt = 0.0
        while not o.foundered()[0] and o.record()[0] < t_max:
            if o.record()[0] >= nxt:
                curve.append(o.readouts())
                nxt += 30.0
            o.step(1)
        curve.append(o.readouts())
        np.testing.assert_array_equal(b.state(i), o.record(), err_msg=f"instance {i}")
        np.testing.assert_array_equal(b.curve(i), np.array(curve), err_msg=f"instance {i} curve")
        assert b.events(i) == o.events()
    b.close()


def test_launch_shape_does_not_change_bits(model):
    ship_p, sim_p, _, sim = model
    ref = None
    shapes = [dict(), dict(team_warps=1, tail_team_warps=0, teams_per_block=1), dict(team_warps=1, teams_per_block=16, blocks=1),
              dict(steps_per_launch=777), dict(team_warps=2), dict(team_warps=4), dict(team_warps=8),
              dict(team_warps=1, tail_team_warps=4, yield_below=20), dict(team_warps=2, tail_team_warps=8, yield_below=20),
              # a whole 16-warp block per simulation, alone and as the last of four phases
              dict(team_warps=16), dict(team_warps=2, tail_team_warps=16, yield_below=20),
              # 4 teams for 20 instances, handing over once 19 remain: the next phase claims the 16 not yet started
              # before the 3 the first phase paused (fewest steps done first), or by index
              dict(team_warps=1, teams_per_block=4, blocks=1, tail_team_warps=4, yield_below=19),
              dict(team_warps=1, teams_per_block=4, blocks=1, tail_team_warps=4, yield_below=19, claim_by_index=True),
              # the caller's claim order for the first phase (last instance first)
              dict(team_warps=1, teams_per_block=4, blocks=1, tail_team_warps=4, yield_below=19, _order=list(range(19, -1, -1))),
              # the column table in every block's shared memory
              dict(stage_columns=True), dict(team_warps=2, tail_team_warps=16, yield_below=20, stage_columns=True),
              dict(steps_per_launch=777, stage_columns=True)]
    for kw in shapes:
        kw = dict(kw)
        order = kw.pop("_order", None)
        b, _ = _perturbed_batch(ship_p, sim_p, sim, 20, "portable", 1800.0, **kw)
        if order is not None:
            b.set_claim_order(order)
        b.run()
        info = b.launch_info()
        ordered = 0 if kw.get("claim_by_index") or kw.get("steps_per_launch") else info["phases"] - 1
        assert info["kernels"] == 1 + info["phases"] + 2 * ordered, kw
        states = np.stack([b.state(i) for i in range(20)])
        steps = [b.summary(i)["steps"] for i in range(20)]
        b.close()
        if ref is None:
            ref = (states, steps)
        else:
            np.testing.assert_array_equal(states, ref[0], err_msg=str(kw))
            assert steps == ref[1]


@pytest.mark.parametrize("numerics", ["portable", "portable32"])
def test_staged_column_table_gives_the_same_bits(model, numerics):
    """Every block copies the column table into its shared memory by bulk asynchronous copies (stage_columns) and the
    buoyancy reads it there: the same states, steps and curves as reading it from global memory, and no block gave up
    waiting for its copy (health 0)."""
    ship_p, sim_p, _, sim = model
    out = []
    for stage in (False, True):
        b, _ = _perturbed_batch(ship_p, sim_p, sim, 40, numerics, 1800.0, curve_every=60.0, stage_columns=stage)
        info = b.launch_info()
        assert (info["staged_phases"] == info["phases"]) if stage else info["staged_phases"] == 0, info
        b.run()
        assert b.health() == 0, (numerics, stage)
        out.append((np.stack([b.state(i) for i in range(40)]), [b.summary(i)["steps"] for i in range(40)], [b.curve(i) for i in range(40)]))
        b.close()
    np.testing.assert_array_equal(out[1][0], out[0][0])
    assert out[1][1] == out[0][1]
    for i in range(40):
        np.testing.assert_array_equal(out[1][2][i], out[0][2][i], err_msg=f"instance {i} curve")
