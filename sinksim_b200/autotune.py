"""Launch-shape autotuner for a batch: times candidate shapes on the batch's own instances and keeps the fastest.

The shape of a run is the team size of its main phase (warps per simulation), the simulations per block and how soon
each phase hands its unfinished instances to the next (larger) team size. The engine picks a shape from the batch
size and the slot size; the fastest one also depends on how uneven the run lengths are, which only running shows.
Every shape gives the same results bit for bit (the engine's launch-shape tests hold them to that), so the tuner
only trades time.

    best, table = tune(make, candidates)

`make(**shape)` returns a ready Batch (instances set) for a shape; each candidate is run `repeats` times after one
warm-up run and scored by its best device time (CUDA events around its launches).

    best, table = search(make)

searches the launch-shape space (DEFAULT_SPACE: main-phase team size, simulations per block, hand-over factor,
last-phase team size, the column table in shared memory) one coordinate at a time from the engine's own choice,
keeping each value that beats the best so far, for up to `rounds` passes over the coordinates; every shape it times is
in the table.
"""

DEFAULT_CANDIDATES = (
    {},                                         # the engine's own choice
    {"team_warps": 1},
    {"team_warps": 2},
    {"team_warps": 4},
    {"handover_factor": 1.0},
    {"handover_factor": 4.0},
    {"team_warps": 2, "handover_factor": 1.0},
)


def tune(make, candidates=DEFAULT_CANDIDATES, repeats=1, log=None):
    """(best shape, [(shape, device ms, sim-steps)]) over `candidates`."""
    table = []
    for shape in candidates:
        b = make(**shape)
        try:
            b.upload()
            b.launch()
            b.download()
            best_ms, steps = None, None
            for _ in range(repeats):
                b.reset()
                b.upload()
                ms = b.launch()
                b.download()
                best_ms = ms if best_ms is None else min(best_ms, ms)
                steps = b.total_steps()
        finally:
            b.close()
        table.append((dict(shape), best_ms, steps))
        if log:
            log(shape, best_ms, steps)
    best = min(table, key=lambda r: r[1])
    return best[0], table


# Values of each launch-shape option the search tries (None: the engine's own choice, the option left unset).
DEFAULT_SPACE = (
    ("team_warps", (None, 1, 2, 4, 8)),
    ("teams_per_block", (None, 2, 4, 8)),
    ("handover_factor", (None, 1.0, 1.5, 3.0, 4.0)),
    ("tail_team_warps", (None, 8)),
    ("stage_columns", (None, True)),
)


def search(make, space=DEFAULT_SPACE, repeats=1, rounds=2, log=None):
    """(best shape, [(shape, device ms, sim-steps)]): coordinate search over `space` from the engine's own choice.

    Each pass tries, for one option at a time, every value of it with the other options at the best shape so far, and
    keeps a value only if it is faster; it stops after `rounds` passes or a pass without change. A shape is timed once
    (the table holds each shape once)."""
    timed = {}
    table = []

    def score(shape):
        key = tuple(sorted(shape.items()))
        if key not in timed:
            _, t = tune(make, candidates=(shape,), repeats=repeats, log=log)
            timed[key] = t[0][1]
            table.append(t[0])
        return timed[key]

    best = {}
    best_ms = score(best)
    for _ in range(rounds):
        changed = False
        for name, values in space:
            for v in values:
                shape = {k: x for k, x in best.items() if k != name}
                if v is not None:
                    shape[name] = v
                if shape == best:
                    continue
                ms = score(shape)
                if ms < best_ms:
                    best, best_ms, changed = shape, ms, True
        if not changed:
            break
    return best, table
