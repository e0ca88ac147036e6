"""The tangent-linear restatement of the step (oracle/sinksim_tangent.cpp), the reference gradient of the adjoint.

Its value part must be the portable step itself: on titanic64 with perturbed connection areas it must reproduce the
C restatement (which is pinned to the reference's golden traces) bit for bit, step after step. Its tangents must be
derivatives: against central differences of the C restatement at a point where no branch of the step switches
within the stencil, over a short horizon, they agree to the differencing error.
"""
import numpy as np

from _support import Oracle, Tangent, load_model, titanic


def _model():
    return load_model(*titanic())


def test_value_part_is_the_portable_step_bit_for_bit():
    ship, sim = _model()
    o, t = Oracle(ship, sim, False), Tangent(ship, sim)
    breach = sim["kindNames"].index("breach")
    for c in np.nonzero(sim["kind"] == breach)[0]:
        a = float(sim["area"][c]) * 1.37
        o.set_connection(int(c), area=a)
        t.set_connection(int(c), area=a)
    for _ in range(6):
        o.step(100)
        t.step(100)
        ro, rt = o.record(), t.record()
        np.testing.assert_array_equal(rt[:7], ro[:7])
        np.testing.assert_array_equal(rt[10:], ro[10:])
        np.testing.assert_array_equal(t.readouts(), o.readouts())


def test_tangents_match_central_differences_on_a_smooth_stretch():
    ship, sim = _model()
    breach = sim["kindNames"].index("breach")
    conns = [int(c) for c in np.nonzero(sim["kind"] == breach)[0] if sim["en"][c]]
    area0 = {c: float(sim["area"][c]) for c in conns}
    steps = 120
    t = Tangent(ship, sim)
    for c in conns:
        t.seed_area(c, 0, area0[c])  # d area / d log-scale of the breach kind
    t.step(steps)
    r, d = t.readouts(tangents=True)

    def run(scale):
        o = Oracle(ship, sim, False)
        for c in conns:
            o.set_connection(c, area=area0[c] * scale)
        o.step(steps)
        return o.readouts()

    h = 1e-6
    fd = (run(np.exp(h)) - run(np.exp(-h))) / (2 * h)
    # trim and the drafts: the tangent and the difference quotient agree to a few parts in a million
    for k in (1, 5, 6):
        assert abs(fd[k] - d[0, k]) <= 1e-5 * abs(d[0, k]) + 1e-12, (k, fd[k], d[0, k])
