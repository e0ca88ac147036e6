"""The adjoint's reverse step (sinksim_b200/csrc/adjoint_step.cuh) run on the CPU by its host harness, against the FP64
tangent-linear restatement of the step (oracle/sinksim_tangent.cpp).

Both differentiate the same branch path of the same portable step; they are a transpose pair, so they must give the
same gradient up to rounding: within 1e-10 relative on titanic64 over 1,000 s of flooding (4,000 steps, merged level
groups, orifices, weirs with the Villemonte factor, the limiter) and on the generated liner over 25 s (single-node level
solves). The objective is the trajectory misfit (squared trim and heave residuals at 8 times) against a target run
at other breach areas.
"""
import numpy as np
import pytest

from _support import Oracle, adjoint_host_gradient, load_model, tangent_gradient, titanic


def _case(ship, sim, steps, scale=1.3, target_scale=1.1):
    nc = len(sim["ca"])
    en = np.array(sim["en"], dtype=np.uint8)
    area = np.array(sim["area"], dtype=np.float64)
    t_on = np.array(sim["tOn"], dtype=np.float64)
    kind = np.asarray(sim["kind"])
    breach = list(sim["kindNames"]).index("breach")
    area[kind == breach] *= scale
    samples = [steps * (k + 1) // 8 for k in range(8)]
    o = Oracle(ship, sim)
    for c in range(nc):
        o.set_connection(c, int(en[c]), float(area[c] * (target_scale if kind[c] == breach else 1.0)), float(t_on[c]))
    trim, heave, done = [], [], 0
    for s in samples:
        o.step(s - done)
        done = s
        r = o.readouts()
        trim.append(r[1])
        heave.append(0.5 * (r[5] + r[6]))
    return en, area, t_on, samples, trim, heave


def _check(ship, sim, steps, tol):
    en, area, t_on, samples, trim, heave = _case(ship, sim, steps)
    J, grad, err = adjoint_host_gradient(ship, sim, en, area, t_on, steps, samples, trim, heave)
    assert err == 0
    nz = [int(c) for c in np.argsort(-np.abs(grad)) if grad[c] != 0]
    assert len(nz) >= 5
    conns = nz[:10]
    Jt, gt = tangent_gradient(ship, sim, en, area, t_on, conns, steps, samples, trim, heave)
    assert J == Jt  # the same forward values, the same sums
    scale = np.max(np.abs(gt))
    for p, c in enumerate(conns):
        assert abs(grad[c] - gt[p]) <= tol * abs(gt[p]) + 1e-13 * scale, (c, grad[c], gt[p])


def test_host_adjoint_equals_tangent_linear_titanic64():
    ship, sim = load_model(*titanic())
    _check(ship, sim, 4000, 1e-10)


def test_host_adjoint_equals_tangent_linear_liner(tmp_path):
    from sinksim_b200 import hullgen

    ship, sim = load_model(*hullgen.write(str(tmp_path)))
    _check(ship, sim, 100, 1e-10)
