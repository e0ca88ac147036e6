"""The adjoint against central differences at h = 1e-6 relative, at points away from regime switches.

"Away from regime switches" is checked, not assumed: the C restatement keeps a digest of every discrete decision of
every step (per node pass the numbers of wet and partial segments, each level update's Newton or bisection branch,
zero and limited flows, clipped volumes, clamped angles; sinksim_oracle.c sso_digest), and a parameter's stencil counts
only when its runs at theta - h, theta and theta + h have the same digest, that is, took the same branch path. On
those stencils the difference quotient and the adjoint must agree to 1e-6 relative (against the gradient's scale).

The gradient workload's parameters on the generated liner (log scales of the door, overflow, deck-opening and
weather-deck-opening connections, areas of the six open breaches), two of its points, the objective at 8 times up to
10 s and up to 25 s of flooding. (Further out the branch path changes within +-1e-6 of the parameters: a difference
quotient there measures jumps, not a derivative.)
"""
import os
import sys
import tempfile

import numpy as np
import pytest

from _support import ROOT, Oracle, load_model
from fdcheck import fd_versus_adjoint

sys.path.insert(0, ROOT)


@pytest.fixture(scope="module")
def liner():
    from sinksim_b200 import hullgen

    return load_model(*hullgen.write(os.path.join(tempfile.gettempdir(), "sinksim_b200_fd_liner")))


@pytest.mark.parametrize("steps", [40, 100])
@pytest.mark.parametrize("point", [0, 1])
def test_adjoint_agrees_with_central_differences_on_one_branch_path(liner, steps, point):
    import bench

    ship, sim = liner
    space = bench.gradient_space(sim)
    samples = [steps * (k + 1) // 8 for k in range(8)]
    o = Oracle(ship, sim)
    for c, a in space.areas(bench.gradient_point(space, -1)).items():
        o.set_connection(c, area=a)
    trim_t, heave_t, done = [], [], 0
    for s in samples:
        o.step(s - done)
        done = s
        r = o.readouts()
        trim_t.append(r[1])
        heave_t.append(0.5 * (r[5] + r[6]))
    theta = bench.gradient_point(space, point)
    J, res = fd_versus_adjoint(ship, sim, space, theta, steps, samples, trim_t, heave_t, h_rel=1e-6)
    scale = max(abs(g) for _, _, g in res)
    checked = [(fd, g) for same, fd, g in res if same]
    assert len(checked) >= 6, f"only {len(checked)} of {len(res)} stencils stayed on one branch path"
    for fd, g in checked:
        assert abs(fd - g) <= 1e-6 * scale, (fd, g, scale)
