"""The launch-shape tuner's selection (sinksim_b200.autotune) with a stand-in batch whose device time depends on
its shape: one warm-up run per candidate, the best of `repeats` timed runs, the fastest shape kept, every batch closed."""
from sinksim_b200.autotune import DEFAULT_CANDIDATES, tune


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
