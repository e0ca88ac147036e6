"""Synthetic batch workloads: the per-instance inputs of the batching benchmarks, seeded and reproducible.

batch_uneven(): the "uneven run length" batch: every instance of one compiled model draws its connection-kind
scale factors from lognormal(0, 0.3), opens each door (kind "door", per door index) with probability 0.2, and runs
until it founders, sinks (|trim| > 15 degrees with the deck edge at the bow under water), settles (|pitch rate| below
1e-5 rad/s for 600 s) or reaches tMax. The rule never changes the physics; it only retires instances.
"""
import math

import numpy as np

SCALED_KINDS = ("breach", "over", "down", "top")


def deck_edge_rule(ship, pitch_deg=15.0, wth=1e-5, settle=600.0):
    """The sink/settle retire rule for a compiled ship: the deck edge at the bow is the top of the most forward
    columns at their largest half-breadth."""
    x = np.asarray(ship["x"])
    front = x >= x.max() - 1e-9
    cols = np.nonzero(front)[0]
    j = cols[np.argmax(np.abs(np.asarray(ship["y"])[cols]))]
    return dict(pitch=math.radians(pitch_deg), x=float(x[j]), y=float(abs(ship["y"][j])), z=float(ship["zhi"][j]), wth=wth, settle=settle)


def batch_uneven(sim, count, seed=20261203, first=0):
    """Per-instance connection settings for instances first .. first+count-1 of the uneven-length batch.

    Returns a list of (area dict {conn: area}, enabled dict {conn: 0/1}); instance i's draws depend only on (seed, i),
    so shards of the batch on several GPUs reproduce the same instances."""
    kinds = list(sim["kindNames"])
    kind = np.asarray(sim["kind"])
    area0 = np.asarray(sim["area"], dtype=np.float64)
    door = kinds.index("door") if "door" in kinds else -1
    door_idx = sorted(set(int(v) for v in np.asarray(sim["idx"])[kind == door])) if door >= 0 else []
    out = []
    for i in range(first, first + count):
        rng = np.random.default_rng([seed, i])
        area, enabled = {}, {}
        for name in SCALED_KINDS:
            if name not in kinds:
                continue
            k = kinds.index(name)
            f = float(rng.lognormal(0.0, 0.3))
            for c in np.nonzero(kind == k)[0]:
                area[int(c)] = float(area0[c] * f)
        for d in door_idx:
            if rng.random() < 0.2:
                for c in np.nonzero((kind == door) & (np.asarray(sim["idx"]) == d))[0]:
                    enabled[int(c)] = 1
        out.append((area, enabled))
    return out
