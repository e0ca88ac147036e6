"""The gradient workload's host side (bench.py --workload gradient): its 10 parameters on the generated liner, seeded
points that do not depend on how the points are split over ranks, and the reference arm's sweep document, whose
instances set exactly the areas the GPU batch is given."""
import json
import math
import sys

import numpy as np

from _support import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402
from sinksim_b200.calibrate import fd_stencil
from sinksim_b200.files import load_model


def _liner():
    ship_p, sim_p = bench.model_paths("liner")
    return load_model(ship_p, sim_p)[1]


def test_space_is_four_kind_scales_and_six_open_breaches():
    sim = _liner()
    sp = bench.gradient_space(sim)
    assert sp.dim == 10 and sp.kinds == ("door", "over", "down", "top")
    names = list(sim["kindNames"])
    assert len(sp.conns) == 6
    for c in sp.conns:
        assert names[int(sim["kind"][c])] == "breach" and int(sim["en"][c]) == 1


def test_points_are_seeded_per_index():
    sp = bench.gradient_space(_liner())
    a = [bench.gradient_point(sp, i) for i in range(-1, 40)]
    b = [bench.gradient_point(sp, i) for i in reversed(range(-1, 40))][::-1]
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    pts = np.stack(a)
    assert np.all(np.abs(pts[:, :4]) < 2.0)               # N(0, 0.3) log scales
    assert np.all((pts[:, 4:] >= 0.1) & (pts[:, 4:] < 0.4))  # U(0.1, 0.4) m2 breach areas
    assert len({tuple(p) for p in pts}) == len(pts)


def test_reference_sweep_sets_the_batch_areas():
    sp = bench.gradient_space(_liner())
    thetas = np.stack([bench.gradient_point(sp, i) for i in range(3)])
    doc = json.loads(json.dumps(bench.gradient_sweep(sp, thetas, 1e-2)))  # as the tool reads it
    cols, areas = sp.area_matrix(fd_stencil(thetas, 1e-2))
    assert len(doc["instances"]) == 3 * 21
    times, every = bench.gradient_times()
    assert doc["tMax"] == times[-1] == 7920.0 and every == 990.0
    for k, inst in enumerate(doc["instances"]):
        assert [o["conn"] for o in inst["connections"]] == cols
        assert [o["area"] for o in inst["connections"]] == areas[k].tolist()
    assert not any(math.isnan(a) for a in areas.ravel())
