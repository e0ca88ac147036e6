"""The GPU adjoint (ssb_adjoint_*, adjoint_kernel.cu) on a B200, through the C ABI.

* Its objective equals the host harness's (the same forward bits: the same values summed in the same order), and its
  gradient with respect to every connection area equals the host harness's run of the same reverse step within 1e-9
  relative (the device sums the pose adjoints in another order), and the FP64 tangent-linear restatement's within
  1e-9 relative, on titanic64 over 1,000 s (4,000 steps, 16 checkpoint segments) and on the generated liner.
* Checkpointing does not change the numbers: intervals of 256, 100 and 4,000 steps give the same bits (the reverse
  of every step runs on the same recomputed tape). Nor does the memory for step records: a ring of one segment (every
  segment recomputed from its checkpoint), one that holds the last few segments of the run (the rest recomputed) and
  one that holds the whole run (nothing recomputed: the phase times show no recomputation) give the same bits.
* Its trim and heave at the sample times equal the batch engine's readout curve records bit for bit.
"""
import numpy as np
import pytest

import sinksim_b200 as ssb
from _support import Oracle, adjoint_host_gradient, load_model, tangent_gradient, titanic

pytestmark = pytest.mark.gpu

SCALES = (1.3, 1.25, 1.35, 1.2)


def _setup(ship, sim, steps, count=len(SCALES)):
    kind = np.asarray(sim["kind"])
    breach = list(sim["kindNames"]).index("breach")
    bconns = np.nonzero(kind == breach)[0].astype(np.int32)
    area0 = np.asarray(sim["area"], dtype=np.float64)
    areas = np.stack([area0[bconns] * SCALES[i % len(SCALES)] for i in range(count)])
    samples = [steps * (k + 1) // 8 for k in range(8)]
    o = Oracle(ship, sim)
    for c in bconns:
        o.set_connection(int(c), area=float(area0[c] * 1.1))
    trim, heave, done = [], [], 0
    for s in samples:
        o.step(s - done)
        done = s
        r = o.readouts()
        trim.append(r[1])
        heave.append(0.5 * (r[5] + r[6]))
    times = [s * sim["dt"] for s in samples]
    return bconns, areas, samples, times, np.array(trim), np.array(heave)


def _run(ship_p, sim_p, ship, sim, steps, k_every=256, count=len(SCALES), tape_budget=0, order=None):
    bconns, areas, samples, times, trim, heave = _setup(ship, sim, steps, count)
    a = ssb.Adjoint(ship_p, sim_p, count=count, t_max=steps * sim["dt"], checkpoint_every=k_every, tape_budget=tape_budget)
    a.set_claim_order(order)
    a.set_connection_areas(0, bconns, areas)
    a.set_objective(times, trim, heave)
    J, g, st, err, ms = a.run()
    tr, hv = a.samples()
    phases, ring, recomputed = a.phase_times(), a.ring_bytes(), a.recomputed_steps()
    a.close()
    return dict(J=J, g=g, steps=st, err=err, trim=tr, heave=hv, bconns=bconns, areas=areas, samples=samples, trimT=trim, heaveT=heave,
                phases=phases, ring=ring, recomputed=recomputed)


def _host(ship, sim, r, i, steps):
    en = np.array(sim["en"], dtype=np.uint8)
    area = np.array(sim["area"], dtype=np.float64)
    area[r["bconns"]] = r["areas"][i]
    t_on = np.array(sim["tOn"], dtype=np.float64)
    return en, area, t_on


@pytest.mark.parametrize("model", ["titanic64", "liner"])
def test_gpu_adjoint_equals_host_adjoint_and_tangent_linear(model, tmp_path):
    if model == "titanic64":
        ship_p, sim_p = titanic()
        steps = 4000
    else:
        from sinksim_b200 import hullgen

        ship_p, sim_p = hullgen.write(str(tmp_path))
        steps = 100
    ship, sim = load_model(ship_p, sim_p)
    r = _run(ship_p, sim_p, ship, sim, steps)
    assert (r["err"] == 0).all()
    assert (r["steps"] == steps).all()
    for i in range(len(SCALES)):
        en, area, t_on = _host(ship, sim, r, i, steps)
        J, g, err = adjoint_host_gradient(ship, sim, en, area, t_on, steps, r["samples"], r["trimT"], r["heaveT"])
        assert err == 0
        assert r["J"][i] == J, (i, r["J"][i], J)
        scale = np.max(np.abs(g))
        np.testing.assert_allclose(r["g"][i], g, rtol=1e-9, atol=1e-12 * scale, err_msg=f"instance {i}")
    # the tangent-linear restatement on instance 0, at the ten largest gradients
    en, area, t_on = _host(ship, sim, r, 0, steps)
    conns = [int(c) for c in np.argsort(-np.abs(r["g"][0]))[:10]]
    Jt, gt = tangent_gradient(ship, sim, en, area, t_on, conns, steps, r["samples"], r["trimT"], r["heaveT"])
    assert Jt == r["J"][0]
    scale = np.max(np.abs(gt))
    for p, c in enumerate(conns):
        assert abs(r["g"][0][c] - gt[p]) <= 1e-9 * abs(gt[p]) + 1e-12 * scale, (c, r["g"][0][c], gt[p])


def test_gpu_adjoint_does_not_depend_on_the_checkpoint_interval():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    base = _run(ship_p, sim_p, ship, sim, 2000, 256, count=2)
    for k in (100, 2000):
        other = _run(ship_p, sim_p, ship, sim, 2000, k, count=2)
        np.testing.assert_array_equal(other["J"], base["J"])
        np.testing.assert_array_equal(other["g"], base["g"], err_msg=f"checkpoints every {k} steps")


def test_gpu_adjoint_does_not_depend_on_the_memory_for_step_records():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    steps, k_every, count = 2000, 100, 2
    whole = _run(ship_p, sim_p, ship, sim, steps, k_every, count=count)
    assert (whole["recomputed"] == 0).all(), whole["recomputed"]
    assert (whole["phases"][:, 1] < 0.01 * whole["phases"][:, 2]).all(), whole["phases"]
    one = _run(ship_p, sim_p, ship, sim, steps, k_every, count=count, tape_budget=1)
    seg = one["ring"]  # one segment of the largest records per team
    assert whole["ring"] > seg
    assert (one["recomputed"] == steps).all(), one["recomputed"]
    some = _run(ship_p, sim_p, ship, sim, steps, k_every, count=count, tape_budget=count * 2 * seg)
    assert some["ring"] == 2 * seg
    # a record is about a third of the largest, so the ring holds the last few of the 20 segments
    assert ((some["recomputed"] > 0) & (some["recomputed"] < steps - 2 * k_every)).all(), some["recomputed"]
    assert (some["recomputed"] % k_every == 0).all()
    # the claim order (last instance first) changes which team takes which instance, not the results
    rev = _run(ship_p, sim_p, ship, sim, steps, k_every, count=count, order=list(range(count - 1, -1, -1)))
    for name, r in (("one segment", one), ("a few segments", some), ("reversed claims", rev)):
        np.testing.assert_array_equal(r["J"], whole["J"], err_msg=name)
        np.testing.assert_array_equal(r["g"], whole["g"], err_msg=name)
        np.testing.assert_array_equal(r["steps"], whole["steps"], err_msg=name)


def test_gpu_adjoint_samples_equal_the_batch_curve():
    ship_p, sim_p = titanic()
    ship, sim = load_model(ship_p, sim_p)
    steps = 2000
    r = _run(ship_p, sim_p, ship, sim, steps, count=2)
    every = r["samples"][0] * sim["dt"]
    with ssb.Batch(ship_p, sim_p, count=2, numerics="portable", t_max=steps * sim["dt"], curve_every=every) as b:
        b.set_connection_areas(0, r["bconns"], r["areas"])
        b.run()
        for i in range(2):
            curve = b.curve(i)  # records at 0, every, 2 every, ...; the last is the final readouts
            trim = curve[1:, 1]
            heave = 0.5 * (curve[1:, 5] + curve[1:, 6])
            np.testing.assert_array_equal(r["trim"][i], trim)
            np.testing.assert_array_equal(r["heave"][i], heave)
