"""The batch run that allocates no device memory (ssb_batch_run_noalloc), through the C ABI.

It serves callers that cannot call cudaMalloc at run time: a host application that owns every device allocation
through its own pool, or code that must not allocate once running. They pass their own device buffers for the
inputs and outputs, and the kernel's scratch lives in a fixed array inside the library. This test holds the results
of two calls in a row, on the same caller buffers refilled with the inputs, to those of the ordinary entry point
(ssb_batch_run) on the same instances, bit for bit (the tolerance of every parity test here): with the batch's plain
options (stops at tMax), with the reference's calm rule (stop 5) and with the sink/settle retire rule
(stops 3 and 4). It also checks that a batch whose scratch would not fit is refused on the host with a clear error
that names the largest count that fits. The file is named so that pytest collects it last.
"""
import os
import re

import numpy as np
import pytest

import sinksim_b200 as ssb
from sinksim_b200.files import decompressed, load_model
from sinksim_b200.workloads import batch_uneven, deck_edge_rule

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _model():
    ship_p = decompressed(os.path.join(GOLDEN, "titanic64.ship.json.gz"))
    sim_p = decompressed(os.path.join(GOLDEN, "titanic.sim.json.gz"))
    return ship_p, sim_p, *load_model(ship_p, sim_p)


def _perturbed(sim, count):
    en = np.tile(sim["en"], (count, 1)).astype(np.uint8)
    area = np.tile(sim["area"], (count, 1)).astype(np.float64)
    breach = sim["kindNames"].index("breach")
    door = sim["kindNames"].index("door")
    for i in range(count):
        area[i, sim["kind"] == breach] *= 1 + 0.03 * i / count
        if i % 3 == 1:
            en[i, np.nonzero(sim["kind"] == door)[0][:4]] = 1
    return en, area


def _calm(sim, count):
    # breaches closed in the even instances (no inflow: the calm rule ends them after 1,800 + 1,200 s), slightly
    # scaled in the odd ones (they flood and run to tMax)
    en, area = _perturbed(sim, count)
    breach = sim["kindNames"].index("breach")
    for i in range(0, count, 2):
        en[i, sim["kind"] == breach] = 0
    return en, area


def _uneven(sim, picks):
    en = np.tile(sim["en"], (len(picks), 1)).astype(np.uint8)
    area = np.tile(sim["area"], (len(picks), 1)).astype(np.float64)
    params = batch_uneven(sim, max(picks) + 1)
    for i, k in enumerate(picks):
        a, e = params[k]
        for c, v in a.items():
            area[i, c] = v
        for c, v in e.items():
            en[i, c] = v
    return en, area


CASES = {
    # name: (batch options, inputs, stop reasons that must occur)
    "plain": (dict(t_max=1500.0), lambda ship, sim: _perturbed(sim, 24), {2}),
    "calm-rule": (dict(t_max=3600.0, stop_when_stable=True), lambda ship, sim: _calm(sim, 8), {5}),
    "retire-rule": (dict(t_max=5 * 3600.0, rule="deck-edge"), lambda ship, sim: _uneven(sim, [0, 1, 2, 7]), {3, 4}),
}


@pytest.mark.parametrize("case", list(CASES))
def test_noalloc_equals_batch_run_on_two_calls(case):
    import torch

    ship_p, sim_p, ship, sim = _model()
    opts, make, stops_wanted = CASES[case]
    opts = dict(opts)
    if opts.get("rule") == "deck-edge":
        opts["rule"] = deck_edge_rule(ship)
    en, area = make(ship, sim)
    count = en.shape[0]
    t_on = np.tile(sim["tOn"], (count, 1)).astype(np.float64)
    nn = len(ship["mu"])

    b = ssb.Batch(ship_p, sim_p, count=count, numerics="portable", **opts)
    for i in range(count):
        for c in range(en.shape[1]):
            if en[i, c] != sim["en"][c]:
                b.set_connection_enabled(i, c, int(en[i, c]))
            if area[i, c] != sim["area"][c]:
                b.set_connection_area(i, c, float(area[i, c]))
    b.run()
    want_state = np.stack([b.state(i) for i in range(count)])
    want_final = np.stack([b.final_readouts(i) for i in range(count)])
    want_steps = [b.summary(i)["steps"] for i in range(count)]
    want_stop = [b.summary(i)["stop"] for i in range(count)]

    dev = torch.device("cuda:0")
    d_en = torch.from_numpy(en).to(dev)
    d_area = torch.from_numpy(area).to(dev)
    d_ton = torch.from_numpy(t_on).to(dev)
    st0 = np.tile(np.array(sim["state0"] + [0.0]), (count, 1))
    d_state = torch.empty((count, 8), dtype=torch.float64, device=dev)
    d_nodes = {k: torch.empty((count, nn), dtype=torch.float64, device=dev) for k in ("vol", "level", "cx", "cy", "cz")}
    d_final = torch.empty((count, 7), dtype=torch.float64, device=dev)
    d_steps = torch.empty(count, dtype=torch.int64, device=dev)
    d_stop = torch.empty(count, dtype=torch.int32, device=dev)
    for call in range(2):
        d_state.copy_(torch.from_numpy(st0))
        for k, src in (("vol", "vol0"), ("level", "level0"), ("cx", "cx0"), ("cy", "cy0"), ("cz", "cz0")):
            d_nodes[k].copy_(torch.from_numpy(np.tile(sim[src], (count, 1))))
        d_final.fill_(np.nan)
        d_steps.fill_(-1)
        d_stop.fill_(-1)
        torch.cuda.synchronize()
        b.run_noalloc(count, d_en.data_ptr(), d_area.data_ptr(), d_ton.data_ptr(), d_state.data_ptr(), d_nodes["vol"].data_ptr(),
                      d_nodes["level"].data_ptr(), d_nodes["cx"].data_ptr(), d_nodes["cy"].data_ptr(), d_nodes["cz"].data_ptr(),
                      d_final.data_ptr(), d_steps.data_ptr(), d_stop.data_ptr(), None)
        torch.cuda.synchronize()
        st = d_state.cpu().numpy()
        np.testing.assert_array_equal(st[:, :7], want_state[:, :7], err_msg=f"{case} call {call}")
        for j, k in enumerate(("vol", "level", "cx", "cy", "cz")):
            np.testing.assert_array_equal(d_nodes[k].cpu().numpy(), want_state[:, 10 + j * nn:10 + (j + 1) * nn],
                                          err_msg=f"{case} call {call} {k}")
        np.testing.assert_array_equal(d_final.cpu().numpy(), want_final, err_msg=f"{case} call {call}")
        assert d_steps.cpu().tolist() == want_steps, f"{case} call {call}"
        stops = [ssb.STOP_REASONS[v] for v in d_stop.cpu().tolist()]
        assert stops == want_stop, f"{case} call {call}"
        assert {ssb.STOP_REASONS[v] for v in stops_wanted} <= set(stops), (case, stops)
    b.close()


def test_noalloc_refuses_a_batch_beyond_its_scratch():
    ship_p, sim_p, _, _ = _model()
    b = ssb.Batch(ship_p, sim_p, count=1, numerics="portable", t_max=60.0)
    with pytest.raises(ssb.SinksimError) as e:
        b.run_noalloc(1_000_000, *([1] * 12), None)
    assert e.value.code == -1 and "scratch" in str(e.value)
    m = re.search(r"at most (\d+) instances", str(e.value))
    assert m and 1000 < int(m.group(1)) < 1_000_000, str(e.value)
    b.close()
