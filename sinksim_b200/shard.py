"""Instance sharding over GPUs: one process per GPU, each running a contiguous block of a batch's instances.

Instances never interact, so a multi-GPU run has no collective inside a step. Rank r steps its own block on its own
GPU; the host gathers the per-rank results (``sinksim.batch-results`` documents) in instance order, and a timing is the
maximum of the ranks' device times. The reference runs a sweep on one GPU (apps/sinksim_cuda_run.cpp:26-83); this is
the layer that spreads the same sweep over the GPUs of a node, launched with one process per GPU (torchrun).
"""
import bisect
import datetime
import itertools
import json
import os
import tempfile

RESULTS_FORMAT = "sinksim.batch-results"


def shard_bounds(count, world, rank, weights=None):
    """(first, n): rank's contiguous block of `count` instances.

    Without weights the blocks differ in size by at most one instance. With weights (expected steps per instance,
    non-negative) the cut between ranks r - 1 and r falls at the first instance whose running weight reaches
    r / world of the total, so the blocks carry about equal work."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of {world}")
    if count < 0:
        raise ValueError(f"count {count}")
    total = None
    if weights is not None:
        w = [float(x) for x in weights]
        if len(w) != count or any(x < 0 for x in w):
            raise ValueError("weights must be one non-negative value per instance")
        total = sum(w)
    if not total:
        base, extra = divmod(count, world)
        first = rank * base + min(rank, extra)
        return first, base + (1 if rank < extra else 0)
    prefix = list(itertools.accumulate(w))
    cuts = [0]
    for r in range(1, world):
        c = bisect.bisect_left(prefix, total * r / world) + 1
        cuts.append(min(max(c, cuts[-1]), count))
    cuts.append(count)
    return cuts[rank], cuts[rank + 1] - cuts[rank]


class Ranks:
    """The ranks of a run: RANK / LOCAL_RANK / WORLD_SIZE from the launcher; a torch.distributed process group when
    there is more than one (nccl on GPUs, gloo for host-only work). Every rank calls the same methods in the same order."""

    def __init__(self, backend="nccl", timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.backend = None
        if self.world > 1:
            import torch.distributed as dist

            if not dist.is_initialized():
                if backend == "nccl":
                    import torch

                    torch.cuda.set_device(self.local)
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.backend = dist.get_backend()

    def _tensor(self, x):
        import torch

        device = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=device)

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, x):
        if not self.dist:
            return x
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.dist:
            return x
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def all_gather(self, values):
        """Every rank's 1-D float64 values concatenated in rank order, on every rank: one all-gather of the lengths,
        one of the values padded to the longest (NCCL on GPUs, gloo on the host)."""
        import numpy as np

        v = np.ascontiguousarray(values, dtype=np.float64).ravel()
        if not self.dist:
            return v.copy()
        import torch

        device = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        n = torch.tensor([v.size], dtype=torch.int64, device=device)
        sizes = [torch.empty_like(n) for _ in range(self.world)]
        self.dist.all_gather(sizes, n)
        lens = [int(s.item()) for s in sizes]
        buf = torch.zeros(max(max(lens), 1), dtype=torch.float64, device=device)
        buf[:v.size] = torch.from_numpy(v).to(device)
        parts = [torch.empty_like(buf) for _ in range(self.world)]
        self.dist.all_gather(parts, buf)
        return np.concatenate([p[:k].cpu().numpy() for p, k in zip(parts, lens)])

    def gather(self, obj):
        """Every rank's object, in rank order, on rank 0 (None on the others)."""
        if not self.dist:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object(obj, out, dst=0)
        return out

    def close(self):
        if self.dist and self.dist.is_initialized():
            self.dist.destroy_process_group()
        self.dist = None


def merge_results(docs):
    """One batch-results document from the ranks' documents of consecutive instance blocks (rank order; None for a
    rank with no instances). The header fields must agree; the instances are concatenated."""
    docs = [d for d in docs if d is not None]
    if not docs:
        raise ValueError("no results to merge")
    head = {k: v for k, v in docs[0].items() if k != "instances"}
    if head.get("format") != RESULTS_FORMAT:
        raise ValueError(f"not a {RESULTS_FORMAT} document")
    for d in docs[1:]:
        for k in ("format", "formatVersion", "ship", "sim", "numerics", "tMax", "every"):
            if d.get(k) != head.get(k):
                raise ValueError(f"the shards' results differ in {k}: {head.get(k)!r} and {d.get(k)!r}")
    out = dict(head)
    out["instances"] = [inst for d in docs for inst in d["instances"]]
    return out


def sweep_size(sweep_path):
    """Instances of a sweep file."""
    from .files import read_json

    return len(read_json(sweep_path)["instances"])


def run_sweep_sharded(ship_path, sim_path, sweep_path, numerics="portable32", results_path=None, ranks=None, weights=None):
    """The sweep on every rank's GPU, each rank taking a contiguous block (balanced by `weights` when given).

    Returns (total steps over the ranks, the maximum of the ranks' wall seconds). Rank 0 writes the merged results."""
    from . import run_sweep_range

    ranks = ranks or Ranks()
    n_total = sweep_size(sweep_path)
    first, n = shard_bounds(n_total, ranks.world, ranks.rank, weights)
    doc, steps, secs = None, 0, 0.0
    if n > 0:
        with tempfile.TemporaryDirectory() as tmp:
            part = os.path.join(tmp, "part.json") if results_path else None
            steps, secs = run_sweep_range(ship_path, sim_path, sweep_path, first, n, numerics, part, ranks.local)
            if part:
                with open(part) as f:
                    doc = json.load(f)
    total_steps = ranks.sum(steps)
    wall = ranks.max(secs)
    if results_path:
        parts = ranks.gather(doc)
        if ranks.rank == 0:
            with open(results_path, "w") as f:
                json.dump(merge_results(parts), f, indent=2)
    return int(total_steps), wall
