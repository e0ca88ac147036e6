"""The drop-in tools on a B200, run the way the reference's own acceptance tests run its tools
(tests/CMakeLists.txt:40-65 of the reference):

* `sinksim_cuda_run --count 8 --precision double|mixed --trace out.json`, then the reference's `sinksim_check` on that
  trace at tolerance 0 in the matching numerics (its cuda_matches_portable / cuda_matches_portable32 tests);
* `sinksim_cuda_run --sweep smoke.sweep.json --precision mixed --results gpu.json` and the reference's CPU sweep of the
  same file, then `sinksim_sweep --compare cpu.json gpu.json` (its sweep_gpu_matches_cpu): RESULT: IDENTICAL, exit 0;
* `sinksim_sweep ... --numerics portable --results` equals the reference's sweep tool value for value;
* the default bounded launches (2,000 steps per launch, as the reference's) and one persistent launch give the same
  trace.
"""
import os
import subprocess

import pytest

from _support import ROOT, fixture, ref_tool, titanic

pytestmark = pytest.mark.gpu

BIN = os.path.join(ROOT, "sinksim_b200", "bin")


def run(cmd, timeout=900):
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    return r


@pytest.mark.parametrize("precision,numerics", [("double", "portable"), ("mixed", "portable32")])
def test_cuda_run_trace_passes_the_reference_checker(tmp_path, precision, numerics):
    ship_p, sim_p = titanic()
    trace = str(tmp_path / f"cuda_titanic.{precision}.trace.json")
    r = run([os.path.join(BIN, "sinksim_cuda_run"), ship_p, sim_p, "--count", "8", "--precision", precision, "--trace", trace])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "steps/s aggregate" in r.stdout and os.path.exists(trace)
    c = run([ref_tool("sinksim_check"), ship_p, sim_p, trace, "--numerics", numerics, "--tol-step", "0", "--tol-window", "0", "--quiet"])
    assert c.returncode == 0, c.stdout + c.stderr


def test_bounded_and_persistent_launches_write_the_same_trace(tmp_path):
    ship_p, sim_p = titanic()
    a, b = str(tmp_path / "bounded.json"), str(tmp_path / "persistent.json")
    common = [os.path.join(BIN, "sinksim_cuda_run"), ship_p, sim_p, "--count", "4", "--precision", "double", "--tmax", "1800"]
    assert run(common + ["--trace", a]).returncode == 0
    assert run(common + ["--steps-per-launch", "0", "--trace", b]).returncode == 0
    assert open(a).read().replace("\n", "") == open(b).read().replace("\n", "")


def test_gpu_sweep_equals_the_reference_cpu_sweep(tmp_path):
    ship_p, sim_p = titanic()
    sweep = fixture("smoke.sweep.json")
    cpu, gpu, gpu2 = str(tmp_path / "sweep.cpu.json"), str(tmp_path / "sweep.gpu.json"), str(tmp_path / "sweep.gpu2.json")
    r = run([ref_tool("sinksim_sweep"), ship_p, sim_p, sweep, "--numerics", "portable32", "--results", cpu])
    assert r.returncode == 0, r.stdout + r.stderr
    g = run([os.path.join(BIN, "sinksim_cuda_run"), ship_p, sim_p, "--sweep", sweep, "--precision", "mixed", "--results", gpu])
    assert g.returncode == 0, g.stdout + g.stderr
    c = run([os.path.join(BIN, "sinksim_sweep"), "--compare", cpu, gpu])
    assert c.returncode == 0 and "RESULT: IDENTICAL" in c.stdout, c.stdout + c.stderr
    # the drop-in sweep tool: the same results file, compared by the reference's own comparer
    s = run([os.path.join(BIN, "sinksim_sweep"), ship_p, sim_p, sweep, "--numerics", "portable32", "--threads", "4", "--results", gpu2])
    assert s.returncode == 0 and "steps/s aggregate" in s.stdout, s.stdout + s.stderr
    c2 = run([ref_tool("sinksim_sweep"), "--compare", cpu, gpu2])
    assert c2.returncode == 0 and "RESULT: IDENTICAL" in c2.stdout, c2.stdout + c2.stderr
