"""Synthetic batch workloads: the per-instance inputs of the batching benchmarks, seeded and reproducible.

batch_uneven(): the "uneven run length" batch: every instance of one compiled model draws four connection-kind
scale factors from lognormal(0, 0.3) (doors, bulkhead overflows, deck openings, weather-deck openings), opens each
door (kind "door", per door index) with probability 0.2, and draws a total breach area U(0.3, 3) m2 spread over the
breaches of its 1-8 most forward breached spaces (random shares; the other breaches closed). It runs until it
founders, sinks (|trim| > 15 degrees with the deck edge at the bow under water), settles (|pitch rate| below 1e-5
rad/s for 600 s) or reaches tMax. The rule never changes the physics; it only retires instances.
"""
import math

import numpy as np

SCALED_KINDS = ("door", "over", "down", "top")
BREACH_TOTAL = (0.3, 3.0)   # m2
BREACH_SPACES = (1, 8)


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
    # breached spaces from the bow: each breach connection's flooded node, ordered by the breach's x (forward first)
    spaces = []
    if "breach" in kinds:
        bk = np.nonzero(kind == kinds.index("breach"))[0]
        for c in sorted(bk, key=lambda c: -float(sim["cx"][c])):
            node = int(sim["cb"][c])
            if node not in spaces:
                spaces.append(node)
        by_space = {s: [int(c) for c in bk if int(sim["cb"][c]) == s] for s in spaces}
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
        if spaces:
            m = int(rng.integers(BREACH_SPACES[0], min(BREACH_SPACES[1], len(spaces)) + 1))
            total = float(rng.uniform(*BREACH_TOTAL))
            open_conns = [c for s in spaces[:m] for c in by_space[s]]
            share = rng.uniform(0.5, 1.5, size=len(open_conns))
            share = share / share.sum()
            for s in spaces[m:]:
                for c in by_space[s]:
                    enabled[c] = 0
            for c, f in zip(open_conns, share):
                area[c] = total * float(f)
                enabled[c] = 1
        out.append((area, enabled))
    return out
