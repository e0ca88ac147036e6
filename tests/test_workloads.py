"""The uneven-run-length batch's inputs (sinksim_b200.workloads): seeded per instance (a shard reproduces its block),
breach totals and spaces, door openings and kind scales with the stated distributions, the sink rule's deck point."""
import math

import numpy as np

from _support import load_model, titanic
from sinksim_b200.workloads import BREACH_SPACES, BREACH_TOTAL, SCALED_KINDS, batch_uneven, deck_edge_rule

N = 2000


def _model():
    return load_model(*titanic())


def test_blocks_reproduce_the_whole_batch():
    _, sim = _model()
    whole = batch_uneven(sim, 40)
    assert batch_uneven(sim, 15, first=20) == whole[20:35]
    assert batch_uneven(sim, 40, seed=7) != whole


def test_breaches_doors_and_scales_follow_their_distributions():
    _, sim = _model()
    kinds = list(sim["kindNames"])
    kind = np.asarray(sim["kind"])
    area0 = np.asarray(sim["area"], dtype=np.float64)
    breach = np.nonzero(kind == kinds.index("breach"))[0]
    # breached spaces from the bow, as the workload orders them
    spaces = []
    for c in sorted(breach, key=lambda c: -float(sim["cx"][c])):
        if int(sim["cb"][c]) not in spaces:
            spaces.append(int(sim["cb"][c]))
    doors = np.nonzero(kind == kinds.index("door"))[0]
    door_ids = sorted(set(int(sim["idx"][c]) for c in doors))
    opened, logs = 0, {k: [] for k in SCALED_KINDS if k in kinds}
    for area, enabled in batch_uneven(sim, N):
        open_breaches = [c for c in breach if enabled.get(int(c), 0) == 1]
        total = sum(area[int(c)] for c in open_breaches)
        assert BREACH_TOTAL[0] - 1e-12 <= total <= BREACH_TOTAL[1] + 1e-12
        hit = sorted(set(int(sim["cb"][c]) for c in open_breaches), key=spaces.index)
        assert BREACH_SPACES[0] <= len(hit) <= BREACH_SPACES[1]
        assert hit == spaces[:len(hit)]  # the most forward ones
        for c in breach:  # every breach of an unselected space is closed
            if int(sim["cb"][c]) not in hit:
                assert enabled.get(int(c)) == 0
        for d in door_ids:
            members = [int(c) for c in doors if int(sim["idx"][c]) == d]
            states = {enabled.get(c, 0) for c in members}
            assert len(states) == 1  # a door opens with all its connections
            opened += states.pop()
        for k in logs:
            members = [int(c) for c in np.nonzero(kind == kinds.index(k))[0] if area0[c] > 0]
            ratios = [area[c] / area0[c] for c in members]
            assert max(ratios) - min(ratios) <= 1e-12 * max(ratios)  # one factor per kind
            logs[k].append(math.log(ratios[0]))
    p = opened / (N * len(door_ids))
    assert abs(p - 0.2) < 0.02
    for k, v in logs.items():
        assert abs(np.mean(v)) < 0.03 and abs(np.std(v) - 0.3) < 0.03, k


def test_deck_edge_point_is_the_bows_widest_column_top():
    ship, _ = _model()
    r = deck_edge_rule(ship)
    x, y, zhi = (np.asarray(ship[k]) for k in ("x", "y", "zhi"))
    front = np.nonzero(x >= x.max() - 1e-9)[0]
    assert r["x"] == x.max() and r["y"] == np.abs(y[front]).max()
    assert r["z"] in zhi[front].tolist()
    assert r["pitch"] == math.radians(15.0) and r["wth"] == 1e-5 and r["settle"] == 600.0
