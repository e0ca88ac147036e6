"""Launch-shape autotuner for a batch: times candidate shapes on the batch's own instances and keeps the fastest.

The shape of a run is the team size of its main phase (warps per simulation), the simulations per block and how soon
each phase hands its unfinished instances to the next (larger) team size. The engine picks a shape from the batch
size and the slot size; the fastest one also depends on how uneven the run lengths are, which only running shows.
Every shape gives the same results bit for bit (the engine's launch-shape tests hold them to that), so the tuner
only trades time.

    best, table = tune(make, candidates)

`make(**shape)` returns a ready Batch (instances set) for a shape; each candidate is run `repeats` times after one
warm-up run and scored by its best device time (CUDA events around its launches).
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
