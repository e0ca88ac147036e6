"""One rank of the gloo sharding test: python tests/_shard_worker.py RANK WORLD PORT OUT_JSON (run by test_shard.py)."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    rank, world, port, out = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
    from sinksim_b200.shard import Ranks, merge_results, shard_bounds

    ranks = Ranks(backend="gloo", timeout_s=60)
    count = 10
    weights = [1, 1, 1, 1, 1, 1, 1, 1, 10, 10]
    first, n = shard_bounds(count, ranks.world, ranks.rank, weights)
    # a fake per-rank results document for this rank's block (what run_sweep_range writes)
    doc = {"format": "sinksim.batch-results", "formatVersion": 1, "ship": "s", "sim": "m", "numerics": "portable",
           "engine": f"rank {rank}", "tMax": 100.0, "every": 0.0,
           "instances": [{"id": f"i{first + k}", "steps": first + k} for k in range(n)]}
    steps = sum(first + k for k in range(n))
    total = ranks.sum(steps)
    slowest = ranks.max(float(rank + 1))
    parts = ranks.gather(doc if n else None)
    ranks.barrier()
    result = {"rank": rank, "first": first, "n": n, "total": total, "max": slowest}
    if rank == 0:
        merged = merge_results(parts)
        result["ids"] = [i["id"] for i in merged["instances"]]
        result["engine"] = merged["engine"]
    ranks.close()
    with open(out, "w") as f:
        json.dump(result, f)


if __name__ == "__main__":
    main()
