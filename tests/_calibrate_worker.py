"""One rank of the gloo calibration sharding test: python tests/_calibrate_worker.py RANK WORLD PORT OUT_JSON (run by
test_calibrate.py). The batch is replaced by a host function, so the ranks' split of each evaluation, the all-gather
of the objective values and the replicated L-BFGS run without a GPU."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


class RosenbrockEvaluator:
    """Stands in for BatchEvaluator: one 'result' per row, the Rosenbrock value of the row."""

    def __init__(self):
        self.rows = 0

    def run(self, thetas):
        import numpy as np

        thetas = np.atleast_2d(thetas)
        self.rows += len(thetas)
        return [{"f": float(np.sum(100.0 * (t[1:] - t[:-1] ** 2) ** 2 + (1.0 - t[:-1]) ** 2))} for t in thetas]


def main():
    rank, world, port, out = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=port)
    import numpy as np

    from sinksim_b200.calibrate import lbfgs_batched, value_and_grad
    from sinksim_b200.shard import Ranks

    ranks = Ranks(backend="gloo", timeout_s=60)

    def objective(inst):
        return inst["f"]

    x0 = np.random.default_rng(5).normal(0.0, 0.5, size=(7, 3))
    ev = RosenbrockEvaluator()
    f_sh, g_sh = value_and_grad(ev, objective, x0, 1e-6, ranks=ranks)
    f_1, g_1 = value_and_grad(RosenbrockEvaluator(), objective, x0, 1e-6)
    rows_first_call = ev.rows
    x, fx, _ = lbfgs_batched(lambda X: value_and_grad(ev, objective, X, 1e-6, ranks=ranks), x0, max_iter=25)
    x1, fx1, _ = lbfgs_batched(lambda X: value_and_grad(RosenbrockEvaluator(), objective, X, 1e-6), x0, max_iter=25)
    parts = ranks.all_gather([] if rank == 1 else [float(rank), 2.5])
    result = {"rank": rank, "rows_first_call": rows_first_call,
              "same_values": bool(np.array_equal(f_sh, f_1) and np.array_equal(g_sh, g_1)),
              "same_lbfgs": bool(np.array_equal(x, x1) and np.array_equal(fx, fx1)), "x": x.tolist(), "parts": parts.tolist()}
    ranks.close()
    with open(out, "w") as f:
        json.dump(result, f)


if __name__ == "__main__":
    main()
