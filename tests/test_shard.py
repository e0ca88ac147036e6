"""Host side of the multi-GPU sweep: the shard cuts, and the reductions and result merging across ranks (two gloo
ranks on the CPU; instances never interact, so no collective runs inside a step)."""
import json
import os
import socket
import subprocess
import sys

import pytest

from sinksim_b200.shard import merge_results, shard_bounds

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("count,world", [(0, 1), (1, 1), (7, 2), (8, 2), (4096, 8), (5, 8), (1000, 3)])
def test_even_shards_cover_the_instances(count, world):
    blocks = [shard_bounds(count, world, r) for r in range(world)]
    assert blocks[0][0] == 0
    for (f0, n0), (f1, _) in zip(blocks, blocks[1:]):
        assert f0 + n0 == f1
    assert sum(n for _, n in blocks) == count
    sizes = [n for _, n in blocks]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_weighted_shards_balance_the_work(world):
    import random

    rng = random.Random(20261203)
    w = [rng.lognormvariate(0, 0.5) * 20000 for _ in range(4096)]
    blocks = [shard_bounds(len(w), world, r, w) for r in range(world)]
    assert blocks[0][0] == 0 and sum(n for _, n in blocks) == len(w)
    for (f0, n0), (f1, _) in zip(blocks, blocks[1:]):
        assert f0 + n0 == f1
    loads = [sum(w[f:f + n]) for f, n in blocks]
    assert max(loads) <= sum(w) / world + max(w)


def test_shard_bounds_rejects_bad_ranks():
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 0, [1.0] * 9)


def test_merge_rejects_mismatched_shards():
    a = {"format": "sinksim.batch-results", "formatVersion": 1, "ship": "s", "sim": "m", "numerics": "portable", "tMax": 1.0,
         "every": 0.0, "instances": [{"id": "a"}]}
    b = dict(a, numerics="portable32", instances=[{"id": "b"}])
    with pytest.raises(ValueError):
        merge_results([a, b])
    assert [i["id"] for i in merge_results([a, None, dict(a, instances=[{"id": "c"}])])["instances"]] == ["a", "c"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_reduce_and_gather(tmp_path):
    port = str(_free_port())
    outs = [tmp_path / f"rank{r}.json" for r in range(2)]
    procs = [subprocess.Popen([sys.executable, os.path.join(HERE, "_shard_worker.py"), str(r), "2", port, str(outs[r])])
             for r in range(2)]
    for p in procs:
        assert p.wait(timeout=180) == 0
    res = [json.loads(o.read_text()) for o in outs]
    # weights 1 x 8 and 10 x 2 (total 28): rank 0 takes instances 0..8 (weight 18 >= 14), rank 1 instance 9
    assert (res[0]["first"], res[0]["n"]) == (0, 9)
    assert (res[1]["first"], res[1]["n"]) == (9, 1)
    assert res[0]["total"] == res[1]["total"] == sum(range(10))
    assert res[0]["max"] == res[1]["max"] == 2.0
    assert res[0]["ids"] == [f"i{k}" for k in range(10)]
    assert res[0]["engine"] == "rank 0"
