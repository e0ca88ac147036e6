"""Calibration host logic: the oracle's objective restated (checked against the reference's own scores of the
reference CPU engine's results), the parameter mapping, the central-difference stencil and the batched L-BFGS."""
import gzip
import json
import math
import os

import numpy as np
import pytest

from _support import GOLDEN, load_model, titanic
from sinksim_b200.calibrate import (ParamSpace, TrajectoryObjective, default_times, fd_reduce, fd_stencil, interpolate, lbfgs_batched,
                                    oracle_objective)


def _obs():
    with open(os.path.join(GOLDEN, "titanic-1912.observations.json")) as f:
        return json.load(f)


def test_oracle_objective_equals_the_reference_scores():
    with open(os.path.join(GOLDEN, "calibration.points.json")) as f:
        pts = json.load(f)
    with gzip.open(os.path.join(GOLDEN, "calibration.results.json.gz"), "rt") as f:
        res = json.load(f)
    obs = _obs()
    for inst, J in zip(res["instances"], pts["J"]):
        assert oracle_objective(inst, obs) == J
    assert abs(pts["J"][0] - 10.4395) < 1e-3  # the compiled model's own values (kind scales 1)


def test_interpolate():
    ts, ys = [0.0, 10.0, 20.0], [1.0, 3.0, 2.0]
    assert interpolate(ts, ys, 5.0) == 2.0
    assert interpolate(ts, ys, 20.0) == 2.0 and interpolate(ts, ys, 25.0, after=7.0) == 7.0
    assert interpolate(ts, ys, 0.0) == 1.0


def test_param_space_is_the_sweep_product():
    _, sim = load_model(*titanic())
    sp = ParamSpace(sim, conns=(3,))
    theta = [0.1, -0.2, 0.05, 0.3, 0.123]
    a = sp.areas(theta)
    kinds = list(sim["kindNames"])
    for c, area in a.items():
        if c == 3:
            assert area == 0.123
            continue
        k = sp.kinds.index(kinds[int(sim["kind"][c])])
        assert area == float(sim["area"][c]) * math.exp(theta[k])
    assert sp.scales(theta) == {k: math.exp(theta[i]) for i, k in enumerate(sp.kinds)}
    with pytest.raises(ValueError):
        sp.areas([0.0])


def test_area_matrix_is_areas_row_by_row():
    _, sim = load_model(*titanic())
    member = int(np.nonzero(np.asarray(sim["kind"]) == list(sim["kindNames"]).index("breach"))[0][0])
    sp = ParamSpace(sim, conns=(3, member))  # a breach set absolutely after its kind's scale, as a sweep override is
    rng = np.random.default_rng(7)
    thetas = np.concatenate([rng.normal(0.0, 0.3, (50, 4)), rng.uniform(0.1, 0.4, (50, 2))], axis=1)
    cols, A = sp.area_matrix(thetas)
    assert A.shape == (50, len(cols))
    for r in range(50):
        d = sp.areas(thetas[r])
        assert list(d) == cols
        assert np.array_equal(np.array(list(d.values())), A[r])  # the same bits
    assert A[:, cols.index(member)].tolist() == thetas[:, 5].tolist()
    with pytest.raises(ValueError):
        sp.area_matrix(np.zeros((2, 3)))


def test_central_differences_of_a_quadratic():
    A = np.array([[3.0, 0.5, 0.0], [0.5, 2.0, 0.1], [0.0, 0.1, 1.0]])
    thetas = np.array([[0.3, -0.2, 1.5], [2.0, 0.1, -3.0]])
    pts = fd_stencil(thetas, 1e-6)
    assert pts.shape == (2 * 7, 3)
    vals = [0.5 * p @ A @ p for p in pts]
    f, g = fd_reduce(thetas, vals, 1e-6)
    assert np.allclose(f, [0.5 * t @ A @ t for t in thetas])
    assert np.allclose(g, thetas @ A, rtol=1e-6, atol=1e-7)


def test_batched_lbfgs_finds_every_rosenbrock_minimum():
    calls = []

    def fg(X):
        calls.append(len(X))
        x, y = X[:, 0], X[:, 1]
        f = (1 - x) ** 2 + 100 * (y - x * x) ** 2
        g = np.stack([-2 * (1 - x) - 400 * x * (y - x * x), 200 * (y - x * x)], axis=1)
        return f, g

    x0 = np.random.default_rng(7).uniform(-2, 2, size=(16, 2))
    x, f, info = lbfgs_batched(fg, x0, max_iter=500, f_target=1e-14)
    assert np.all(f < 1e-12), f
    assert np.allclose(x, 1.0, atol=1e-6)
    assert info["evaluations"] == len(calls) and max(calls) == 16


def test_trajectory_objective():
    times = default_times()
    assert len(times) == 8 and times[0] == 990.0 and times[-1] == 7920.0
    t = [990.0 * k for k in range(9)]
    inst = {"curve": {"t": t, "trim": [0.01 * k for k in range(9)], "draftF": [10 + 0.1 * k for k in range(9)],
                      "draftA": [10.0] * 9}}
    obj = TrajectoryObjective.from_target(inst, times)
    assert obj(inst) == 0.0
    other = {"curve": dict(inst["curve"], trim=[0.02 * k for k in range(9)])}
    assert obj(other) == pytest.approx(sum((0.01 * k) ** 2 for k in range(1, 9)))


def test_two_gloo_ranks_split_the_stencil_and_agree(tmp_path):
    import socket
    import subprocess
    import sys

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = str(s.getsockname()[1])
    here = os.path.dirname(os.path.abspath(__file__))
    outs = [tmp_path / f"rank{r}.json" for r in range(2)]
    procs = [subprocess.Popen([sys.executable, os.path.join(here, "_calibrate_worker.py"), str(r), "2", port, str(outs[r])])
             for r in range(2)]
    for p in procs:
        assert p.wait(timeout=180) == 0
    res = [json.loads(o.read_text()) for o in outs]
    # 7 points x (2 x 3 + 1) = 49 stencil runs: 25 on rank 0, 24 on rank 1
    assert [r["rows_first_call"] for r in res] == [25, 24]
    assert all(r["same_values"] and r["same_lbfgs"] for r in res)  # the same bits as one process, on every rank
    assert res[0]["x"] == res[1]["x"]
    assert res[0]["parts"] == res[1]["parts"] == [0.0, 2.5]  # rank 1 sent nothing


def test_lbfgs_device_minimises_a_batch_of_quadratics():
    """The device L-BFGS (torch tensors; here on the CPU) drives every restart of a badly scaled quadratic to its
    minimum, and stops a restart once its relative target is met."""
    import torch

    from sinksim_b200.calibrate import lbfgs_device

    rng = np.random.default_rng(3)
    A = np.diag([1.0, 10.0, 100.0, 0.5])
    xs = rng.normal(size=(6, 4))

    def fg(X):
        d = X - torch.as_tensor(xs, dtype=torch.float64)
        Ad = d @ torch.as_tensor(A)
        return (d * Ad).sum(1), 2 * Ad

    x0 = np.zeros((6, 4))
    x, f, info = lbfgs_device(fg, x0, max_iter=60, device="cpu")
    assert float(f.max()) < 1e-12
    np.testing.assert_allclose(x.numpy(), xs, atol=1e-6)
    x, f, info = lbfgs_device(fg, x0, max_iter=60, rel_target=1e-4, device="cpu")
    assert bool((f <= 1e-4 * info["f0"]).all())
