"""The batch run that allocates no device memory (ssb_batch_run_noalloc), through the C ABI.

It serves callers that cannot call cudaMalloc at run time: a host application that owns every device allocation
through its own pool, or code that must not allocate once running. They pass their own device buffers for the
inputs and outputs, and the kernel's scratch lives in a fixed array inside the library. This test holds the results
of two calls in a row, on the same caller buffers refilled with the inputs, to those of the ordinary entry point
(ssb_batch_run) on the same instances, bit for bit (the tolerance of every parity test here). It also checks that a
batch whose scratch would not fit is refused on the host with a clear error. The file is named so that pytest
collects it last.
"""
import os

import numpy as np
import pytest

import sinksim_b200 as ssb
from sinksim_b200.files import decompressed, load_model

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _inputs(sim, count):
    nc = len(sim["ca"])
    en = np.tile(sim["en"], (count, 1)).astype(np.uint8)
    area = np.tile(sim["area"], (count, 1)).astype(np.float64)
    t_on = np.tile(sim["tOn"], (count, 1)).astype(np.float64)
    breach = sim["kindNames"].index("breach")
    door = sim["kindNames"].index("door")
    for i in range(count):
        area[i, sim["kind"] == breach] *= 1 + 0.03 * i / count
        if i % 3 == 1:
            en[i, np.nonzero(sim["kind"] == door)[0][:4]] = 1
    assert en.shape == (count, nc)
    return en, area, t_on


def test_noalloc_equals_batch_run_on_two_calls():
    import torch

    ship_p = decompressed(os.path.join(GOLDEN, "titanic64.ship.json.gz"))
    sim_p = decompressed(os.path.join(GOLDEN, "titanic.sim.json.gz"))
    ship, sim = load_model(ship_p, sim_p)
    count, t_max = 24, 1500.0
    en, area, t_on = _inputs(sim, count)
    nn = len(ship["mu"])

    b = ssb.Batch(ship_p, sim_p, count=count, numerics="portable", t_max=t_max)
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
        torch.cuda.synchronize()
        b.run_noalloc(count, d_en.data_ptr(), d_area.data_ptr(), d_ton.data_ptr(), d_state.data_ptr(), d_nodes["vol"].data_ptr(),
                      d_nodes["level"].data_ptr(), d_nodes["cx"].data_ptr(), d_nodes["cy"].data_ptr(), d_nodes["cz"].data_ptr(),
                      d_final.data_ptr(), d_steps.data_ptr(), d_stop.data_ptr(), None)
        torch.cuda.synchronize()
        st = d_state.cpu().numpy()
        np.testing.assert_array_equal(st[:, :7], want_state[:, :7], err_msg=f"call {call}")
        for j, k in enumerate(("vol", "level", "cx", "cy", "cz")):
            np.testing.assert_array_equal(d_nodes[k].cpu().numpy(), want_state[:, 10 + j * nn:10 + (j + 1) * nn], err_msg=f"call {call} {k}")
        np.testing.assert_array_equal(d_final.cpu().numpy(), want_final, err_msg=f"call {call}")
        assert d_steps.cpu().tolist() == want_steps
        assert set(d_stop.cpu().tolist()) <= {1, 2}
    b.close()


def test_noalloc_refuses_a_batch_beyond_its_scratch():
    ship_p = decompressed(os.path.join(GOLDEN, "titanic64.ship.json.gz"))
    sim_p = decompressed(os.path.join(GOLDEN, "titanic.sim.json.gz"))
    b = ssb.Batch(ship_p, sim_p, count=1, numerics="portable", t_max=60.0)
    with pytest.raises(ssb.SinksimError) as e:
        b.run_noalloc(1_000_000, *([1] * 12), None)
    assert e.value.code == -1 and "scratch" in str(e.value)
    b.close()
