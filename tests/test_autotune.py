"""The launch-shape tuner's selection (sinksim_b200.autotune) with a stand-in batch whose device time depends on
its shape: one warm-up run per candidate, the best of `repeats` timed runs, the fastest shape kept, every batch closed."""
from sinksim_b200.autotune import DEFAULT_CANDIDATES, search, tune


class FakeBatch:
    def __init__(self, times, log, **shape):
        self.key = tuple(sorted(shape.items()))
        self.times = list(times[self.key])
        self.log = log
        self.closed = False

    def upload(self):
        pass

    def launch(self):
        self.log.append(self.key)
        return self.times.pop(0)

    def download(self):
        pass

    def reset(self):
        pass

    def total_steps(self):
        return 1000

    def close(self):
        self.closed = True


def test_tune_keeps_the_fastest_shape():
    times = {tuple(sorted(c.items())): [99.0, 10.0 + k, 9.0 + k] for k, c in enumerate(DEFAULT_CANDIDATES)}
    times[(("team_warps", 4),)] = [1.0, 8.5, 3.0]  # fastest at its best timed run; the warm-up run is not counted
    made, log = [], []

    def make(**shape):
        b = FakeBatch(times, log, **shape)
        made.append(b)
        return b

    best, table = tune(make, repeats=2)
    assert best == {"team_warps": 4}
    assert [r[0] for r in table] == [dict(c) for c in DEFAULT_CANDIDATES]
    assert dict((tuple(sorted(s.items())), ms) for s, ms, _ in table)[(("team_warps", 4),)] == 3.0
    assert all(steps == 1000 for _, _, steps in table)
    assert len(log) == 3 * len(DEFAULT_CANDIDATES)  # one warm-up and two timed launches each
    assert all(b.closed for b in made)


class CostBatch:
    """A batch whose device time is a function of its shape (every launch the same)."""

    def __init__(self, cost, log, **shape):
        self.ms = cost(shape)
        self.log = log
        self.shape = dict(shape)

    def upload(self):
        pass

    def launch(self):
        self.log.append(tuple(sorted(self.shape.items())))
        return self.ms

    def download(self):
        pass

    def reset(self):
        pass

    def total_steps(self):
        return 1000

    def close(self):
        pass


def test_search_descends_one_option_at_a_time():
    # fastest at team_warps=2, teams_per_block=4, handover_factor=1.5; the column table in shared memory is slower
    def cost(shape):
        ms = 100.0
        ms += {None: 20, 1: 30, 2: 0, 4: 10, 8: 40}[shape.get("team_warps")]
        ms += {None: 5, 2: 8, 4: 0, 8: 3}[shape.get("teams_per_block")]
        ms += {None: 4, 1.0: 6, 1.5: 0, 3.0: 2, 4.0: 3}[shape.get("handover_factor")]
        ms += 10 if shape.get("stage_columns") else 0
        ms += 1 if shape.get("tail_team_warps") == 8 else 0
        return ms

    log = []
    best, table = search(lambda **s: CostBatch(cost, log, **s))
    assert best == {"team_warps": 2, "teams_per_block": 4, "handover_factor": 1.5}
    keys = [tuple(sorted(s.items())) for s, _, _ in table]
    assert len(keys) == len(set(keys))  # every shape timed once
    assert min(ms for _, ms, _ in table) == cost(best)
    assert keys[0] == ()  # the engine's own choice first
