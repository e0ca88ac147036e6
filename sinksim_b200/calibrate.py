"""Calibration on the batch engine: objectives over instance results, many parameter points per GPU launch.

* The reference's calibration driver (tools/py/calibrate_gpu.py): the oracle's objective against the 1912
  observations (trim, list, founder time, event times) and its batched random search over connection-kind scales,
  one GPU batch per round.
* Gradient calibration on the plain batched engine: a trajectory objective (squared trim and heave residuals at fixed
  times against a target trajectory), gradients by central finite differences with every point's 2 P + 1 runs in
  one batch, batched L-BFGS over many restarts, and a torch.autograd.Function whose backward returns those gradients.

Parameters are a vector theta: log scale factors on connection kinds (area = compiled area x exp(theta_k) for every
connection of kind k: the single product of sweep::apply's kind scale, engine/include/sinksim/sweep.hpp:49-65, so a
point here and the same scales in a sweep file give the same bits) followed by absolute areas (m2) of chosen
connections, set after the kind scales as a sweep's connection overrides are.

    python -m sinksim_b200.calibrate search  --observations obs.json [--rounds 5 --batch 264 --span 0.3]
    python -m sinksim_b200.calibrate lbfgs   [--restarts 64 --iters 30 --seed 1]
    torchrun --nproc-per-node N -m sinksim_b200.calibrate lbfgs ...   (each evaluation's runs spread over N GPUs)
"""
import argparse
import json
import math
import os
import random
import sys
import time

import numpy as np

KIND_PARAMS = ("breach", "over", "down", "top")
CURVE_COLUMNS = ("t", "trim", "list", "water", "inflow", "draftF", "draftA")


class ParamSpace:
    """theta -> per-connection areas for one compiled sim."""

    def __init__(self, sim, kinds=KIND_PARAMS, conns=()):
        names = list(sim["kindNames"])
        missing = [k for k in kinds if k not in names]
        if missing:
            raise ValueError(f"connection kinds {missing} are not in this sim ({names})")
        kind = np.asarray(sim["kind"])
        self.kinds = tuple(kinds)
        self.conns = tuple(int(c) for c in conns)
        self.area0 = [float(a) for a in sim["area"]]
        self.members = [[int(c) for c in np.nonzero(kind == names.index(k))[0]] for k in self.kinds]
        n = len(self.area0)
        if any(not 0 <= c < n for c in self.conns):
            raise ValueError("connection index out of range")

    @property
    def dim(self):
        return len(self.kinds) + len(self.conns)

    def areas(self, theta):
        """{connection: area} of one point (only the connections theta touches)."""
        theta = [float(v) for v in theta]
        if len(theta) != self.dim:
            raise ValueError(f"theta has {len(theta)} values, the space {self.dim}")
        out = {}
        for k, members in enumerate(self.members):
            factor = math.exp(theta[k])
            for c in members:
                out[c] = self.area0[c] * factor
        for j, c in enumerate(self.conns):
            out[c] = theta[len(self.kinds) + j]
        return out

    def area_matrix(self, thetas):
        """(connections, areas [M, len(connections)]): areas(row) of every row of thetas as one array, with the same
        values bit for bit (one exp per point and kind, then the single product per connection)."""
        thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
        if thetas.shape[1] != self.dim:
            raise ValueError(f"theta has {thetas.shape[1]} values, the space {self.dim}")
        cols, index = [], {}
        for c in [c for members in self.members for c in members] + list(self.conns):
            if c not in index:
                index[c] = len(cols)
                cols.append(c)
        out = np.empty((thetas.shape[0], len(cols)))
        area0 = np.asarray(self.area0)
        for k, members in enumerate(self.members):
            factor = np.array([math.exp(float(v)) for v in thetas[:, k]])
            out[:, [index[c] for c in members]] = area0[members][None, :] * factor[:, None]
        for j, c in enumerate(self.conns):
            out[:, index[c]] = thetas[:, len(self.kinds) + j]
        return cols, out

    def scales(self, theta):
        """The kind-scale factors of one point, as a sweep instance's "scale" would hold them."""
        return {k: math.exp(float(theta[i])) for i, k in enumerate(self.kinds)}


class InstanceResult(dict):
    """One instance's results in the batch-results layout: curve (columns of the readout curve), foundered,
    founderT, events ([{t, id}]) and steps."""


def _results_from_batch(batch, sim_doc, count):
    mon_ids = list(sim_doc["monitors"]["id"])
    mark_ids = list(sim_doc["marks"]["id"])
    out = []
    for i in range(count):
        s = batch.summary(i)
        rec = batch.curve(i)
        curve = {name: [float(v) for v in rec[:, j]] for j, name in enumerate(CURVE_COLUMNS)}
        events = []
        for t, ident, kind in batch.events(i):
            events.append({"t": t, "id": mon_ids[ident] if kind == 0 else mark_ids[ident] if kind == 1 else "founder"})
        out.append(InstanceResult(curve=curve, foundered=s["foundered"], founderT=s["founder_t"], events=events,
                                  steps=s["steps"]))
    return out


class BatchEvaluator:
    """Runs parameter points of one model as the instances of one GPU batch."""

    def __init__(self, ship_path, sim_path, space=None, numerics="portable", t_max=5 * 3600.0, curve_every=30.0, device=0,
                 rule=None, stop_when_stable=False):
        from .files import load_model, read_json

        self.ship_path, self.sim_path = ship_path, sim_path
        _, self.sim = load_model(ship_path, sim_path)
        self.sim_doc = read_json(sim_path)
        self.space = space or ParamSpace(self.sim)
        self.numerics, self.t_max, self.curve_every, self.device = numerics, float(t_max), float(curve_every), device
        self.rule, self.stop_when_stable = rule, stop_when_stable
        self.runs = 0
        self.instances = 0
        self.device_ms = 0.0

    def run(self, thetas):
        """Results of every row of thetas ([M, dim]), in order."""
        from . import Batch

        thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
        m = thetas.shape[0]
        b = Batch(self.ship_path, self.sim_path, count=m, numerics=self.numerics, traced_instances=0, t_max=self.t_max,
                  curve_every=self.curve_every, device=self.device, rule=self.rule, stop_when_stable=self.stop_when_stable)
        try:
            cols, areas = self.space.area_matrix(thetas)
            if cols:
                b.set_connection_areas(0, cols, areas)
            b.upload()
            ms = b.launch()
            self.device_ms += ms
            b.download()
            res = _results_from_batch(b, self.sim_doc, m)
            # the last batch's shape and counts, for callers that report them (device ms, sim-steps, launch phases,
            # bytes moved between host and device)
            self.last = {"device_ms": ms, "steps": b.total_steps(), "phases": b.phase_stats(), "launch": b.launch_info(),
                         "transfer": b.transfer_bytes()}
        finally:
            b.close()
        self.runs += 1
        self.instances += m
        return res


# ------------------------------------------------------------------------------------------ objectives

def interpolate(ts, ys, t, after=None):
    """Linear interpolation of a curve column at time t (s); past the last record its value (or `after`). The
    oracle's calibration reads its curves this way (tools/py/sweep.py:93-103)."""
    if t >= ts[-1]:
        return ys[-1] if after is None else after
    for i in range(1, len(ts)):
        if ts[i] >= t:
            frac = (t - ts[i - 1]) / (ts[i] - ts[i - 1])
            return ys[i - 1] + frac * (ys[i] - ys[i - 1])
    return ys[0]


def oracle_terms(inst, obs):
    """The residual terms of the oracle's calibration objective (tools/py/calibrate_gpu.py:35-64) in its order:
    (weight, residual / sigma) for each trim point after minute 0, the founder time, each list point and each event
    (an event that did not happen counts at the founder time; an instance still afloat founders at afloatFounderMin)."""
    ob = obs["objective"]
    curve = inst["curve"]
    sank = bool(inst["foundered"])
    founder_min = inst["founderT"] / 60 if sank else ob["afloatFounderMin"]
    founder_s = inst["founderT"] if sank else 1e9
    terms = []
    for p in obs["trim"]:
        minute = p["min"]
        if minute == 0:
            continue
        sigma = next(band["sigma"] for band in ob["trimSigmaByMinute"] if minute <= band["upTo"])
        model = ob["trimAfterFounder"] if minute * 60 > founder_s else interpolate(curve["t"], curve["trim"], minute * 60)
        terms.append((1.0, (model - p["deg"]) / sigma))
    terms.append((1.0, (founder_min - obs["founderMin"]) / ob["founderSigmaMin"]))
    for p in obs["list"]:
        minute = p["min"]
        model = ob["listAfterFounder"] if minute * 60 > founder_s else interpolate(curve["t"], curve["list"], minute * 60)
        terms.append((ob["listWeight"], (model - p["deg"]) / ob["listSigmaDeg"]))
    seen = {}
    for e in inst["events"]:
        seen[e["id"]] = e["t"] / 60
    for e in ob["events"]:
        terms.append((1.0, (seen.get(e["id"], founder_min) - e["obsMin"]) / e["sigmaMin"]))
    return terms


def oracle_objective(inst, obs):
    """J = sum of weight x (residual / sigma)^2 over oracle_terms, accumulated in order from 0."""
    total = 0.0
    for w, r in oracle_terms(inst, obs):
        total += r ** 2 if w == 1.0 else w * r ** 2
    return total


class TrajectoryObjective:
    """Sum of squared trim (deg) and heave (m) residuals at fixed times against a target trajectory.

    Heave is the mean of the forward and aft drafts of the readouts. The curve is recorded every `every` seconds and
    the times are multiples of it, so each value is a record's; an instance that stopped earlier holds its last
    record."""

    def __init__(self, times, trim, heave):
        self.times = [float(t) for t in times]
        self.trim = [float(v) for v in trim]
        self.heave = [float(v) for v in heave]

    @staticmethod
    def sample(inst, times):
        c = inst["curve"]
        heave_curve = [0.5 * (f + a) for f, a in zip(c["draftF"], c["draftA"])]
        return ([interpolate(c["t"], c["trim"], t) for t in times], [interpolate(c["t"], heave_curve, t) for t in times])

    @classmethod
    def from_target(cls, inst, times):
        trim, heave = cls.sample(inst, times)
        return cls(times, trim, heave)

    def __call__(self, inst):
        trim, heave = self.sample(inst, self.times)
        total = 0.0
        for k in range(len(self.times)):
            total += (trim[k] - self.trim[k]) ** 2 + (heave[k] - self.heave[k]) ** 2
        return total


def default_times(t_end=7920.0, n=8):
    """n equally spaced times ending at t_end (s): 990 s apart for 8 times in 2.2 h (7,920 s)."""
    return [t_end * (k + 1) / n for k in range(n)]


# ------------------------------------------------------------------------------------------ gradients

# The simulated objectives are smooth only at coarse scales: connection limiters switch, Newton iteration counts and
# threshold crossings change from one parameter value to the next, so central differences with relative steps of 1e-4
# and below are noise (on titanic64, 1.1 h trajectory: a derivative of about -7 at steps of 1e-2 and 1e-3 reads -15 at
# 1e-4, -76 at 1e-6 and 2e4 at 1e-8). The default step is 1e-2.
DEFAULT_FD_STEP = 1e-2


def fd_steps(theta, h_rel):
    """Central-difference step per parameter: h_rel x max(|theta_i|, 1)."""
    return h_rel * np.maximum(np.abs(theta), 1.0)


def fd_stencil(thetas, h_rel):
    """The points of central differences around each row of thetas ([R, P]): rows [R x (2 P + 1), P], per point its
    centre, then +h and -h along each parameter in turn."""
    thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
    r, p = thetas.shape
    out = np.empty((r, 2 * p + 1, p))
    for i in range(r):
        h = fd_steps(thetas[i], h_rel)
        out[i, 0] = thetas[i]
        for j in range(p):
            out[i, 1 + 2 * j] = thetas[i]
            out[i, 1 + 2 * j, j] += h[j]
            out[i, 2 + 2 * j] = thetas[i]
            out[i, 2 + 2 * j, j] -= h[j]
    return out.reshape(r * (2 * p + 1), p)


def fd_reduce(thetas, values, h_rel):
    """Objective and central-difference gradient per point from the stencil's objective values."""
    thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
    r, p = thetas.shape
    v = np.asarray(values, dtype=np.float64).reshape(r, 2 * p + 1)
    f = v[:, 0].copy()
    g = np.empty((r, p))
    for i in range(r):
        h = fd_steps(thetas[i], h_rel)
        # (theta + h) - (theta - h) as the stencil rounded it
        for j in range(p):
            span = (thetas[i, j] + h[j]) - (thetas[i, j] - h[j])
            g[i, j] = (v[i, 1 + 2 * j] - v[i, 2 + 2 * j]) / span
    return f, g


def value_and_grad(evaluator, objective, thetas, h_rel=DEFAULT_FD_STEP, ranks=None):
    """Objective and its central-difference gradient at every row of thetas, all from one batch.

    With `ranks` (sinksim_b200.shard.Ranks) of several processes, one per GPU, each rank runs a contiguous block of
    the stencil's runs and the objective values are all-gathered (one collective per call), so every rank returns the
    same values and gradients and an optimiser replicated on the ranks takes the same steps on each."""
    pts = fd_stencil(thetas, h_rel)
    if ranks is None or ranks.world == 1:
        vals = [objective(inst) for inst in evaluator.run(pts)]
    else:
        from .shard import shard_bounds

        first, n = shard_bounds(len(pts), ranks.world, ranks.rank)
        mine = [objective(inst) for inst in evaluator.run(pts[first:first + n])] if n else []
        vals = ranks.all_gather(mine)
    return fd_reduce(thetas, vals, h_rel)


# ------------------------------------------------------------------------------------------ the configurations' parameters

WORKLOAD_KINDS = ("door", "over", "down", "top")
WORKLOAD_BREACHES = 6
WORKLOAD_SEED = 20261205


def workload_space(sim):
    """The 10 parameters of the gradient and calibration configurations: log scale factors of the door, overflow,
    deck-opening and weather-deck-opening connections, then the areas (m2) of the first six open breaches."""
    names = list(sim["kindNames"])
    kind, en = np.asarray(sim["kind"]), np.asarray(sim["en"])
    breaches = np.nonzero((kind == names.index("breach")) & (en != 0))[0][:WORKLOAD_BREACHES]
    return ParamSpace(sim, kinds=WORKLOAD_KINDS, conns=[int(c) for c in breaches])


def workload_point(space, i, seed=WORKLOAD_SEED):
    """Point i of the seeded stream (i = -1: the hidden point behind the target trajectory): kind log scales N(0, 0.3)
    (lognormal(0, 0.3) factors), breach areas U(0.1, 0.4) m2. Each point has its own generator, so a block of points
    does not depend on how many there are."""
    rng = np.random.default_rng([seed, i + 1])
    nk = len(space.kinds)
    return np.concatenate([rng.normal(0.0, 0.3, nk), rng.uniform(0.1, 0.4, space.dim - nk)])


# ------------------------------------------------------------------------------------------ gradients by the adjoint

class AdjointEvaluator:
    """Objective and gradient of a TrajectoryObjective at many parameter points, by the engine's hand-written discrete
    adjoint (sinksim_b200.Adjoint: the FP64 step reversed from the forward run's packed step records, kept in device
    memory; checkpoints every `checkpoint_every` steps, and recomputation from them of what the memory does not hold). One call runs every point forward and back on the GPU: 1 gradient per instance instead of the 2 P + 1
    runs of central differences.

    The adjoint returns d J / d area[c] for every connection; the chain rule to theta is exact: a kind's log scale
    moves the area of each of its connections by area[c] per unit (area = compiled area x exp(theta_k)), an absolute
    area parameter moves its connection's area one for one (and takes that connection out of its kind's sum, as it
    overrides the scaled area)."""

    def __init__(self, ship_path, sim_path, space=None, t_max=7920.0, device=0, checkpoint_every=256, tape_budget=0, team_warps=0):
        from .files import load_model

        self.ship_path, self.sim_path = ship_path, sim_path
        _, self.sim = load_model(ship_path, sim_path)
        self.space = space or ParamSpace(self.sim)
        self.t_max, self.device, self.k, self.tape_budget, self.team_warps = float(t_max), device, checkpoint_every, tape_budget, team_warps
        self._adj = None
        self._steps = None
        self.device_ms = 0.0
        self.instances = 0
        self.last = None

    def _engine(self, count):
        from . import Adjoint

        if self._adj is None or self._adj.count != count:
            if self._adj is not None:
                self._adj.close()
            self._adj = Adjoint(self.ship_path, self.sim_path, count=count, t_max=self.t_max, checkpoint_every=self.k, device=self.device,
                                tape_budget=self.tape_budget, team_warps=self.team_warps)
        return self._adj

    def close(self):
        if self._adj is not None:
            self._adj.close()
            self._adj = None

    def value_and_grad(self, thetas, objective):
        """(f [R], g [R, P], steps [R]) at the rows of thetas for `objective` (a TrajectoryObjective)."""
        thetas = np.atleast_2d(np.asarray(thetas, dtype=np.float64))
        r = thetas.shape[0]
        a = self._engine(r)
        cols, areas = self.space.area_matrix(thetas)
        a.set_connection_areas(0, cols, areas)
        a.set_objective(objective.times, objective.trim, objective.heave)
        # the previous call's run lengths (nearby points in an optimisation loop) order the claims, longest first
        a.set_claim_order(None if self._steps is None or self._steps.size != r else np.argsort(-self._steps, kind="stable"))
        J, G, steps, err, ms = a.run()
        self._steps = np.asarray(steps, dtype=np.int64).copy()
        if np.any(err):
            raise RuntimeError(f"the adjoint took a branch it does not differentiate in {int(np.count_nonzero(err))} instances (bits {sorted(set(err.tolist()))})")
        self.device_ms += ms
        self.instances += r
        ph = a.phase_times()
        self.last = {"device_ms": ms, "steps": int(steps.sum()), "info": a.info(), "recomputed": int(a.recomputed_steps().sum()),
                     "phase_team_s": [float(v) for v in ph.sum(0)], "ring_bytes": a.ring_bytes()}
        col_of = {c: j for j, c in enumerate(cols)}
        g = np.zeros((r, self.space.dim))
        overridden = set(self.space.conns)
        for k, members in enumerate(self.space.members):
            for c in members:
                if c not in overridden:
                    g[:, k] += G[:, c] * areas[:, col_of[c]]
        nk = len(self.space.kinds)
        for j, c in enumerate(self.space.conns):
            g[:, nk + j] = G[:, c]
        return J, g, steps


# ------------------------------------------------------------------------------------------ optimisers

def lbfgs_batched(fg, x0, max_iter=50, memory=8, f_target=None, rel_tol=1e-12, c1=1e-4, max_backtracks=12, callback=None, max_step=None):
    """L-BFGS on many independent starting points at once; fg(X [K, P]) -> (f [K], g [K, P]) evaluates all of its rows
    in one call (one GPU batch).

    Each iteration evaluates every active point's trial step together; a point whose trial fails the Armijo test
    halves its step and retries in the next call. A point stops when f <= f_target, when its relative decrease falls
    below rel_tol, or after max_iter iterations. With max_step, a trial step is at most that long (Euclidean, in
    parameter units): curvature pairs from a rough objective can make the quasi-Newton direction very long. Returns
    (x, f, info) with info = {iterations, evaluations, history: [best f after each call]}."""
    x = np.array(x0, dtype=np.float64, copy=True)
    r, p = x.shape
    f, g = fg(x)
    f = np.asarray(f, dtype=np.float64)
    g = np.asarray(g, dtype=np.float64)
    S = [[] for _ in range(r)]
    Y = [[] for _ in range(r)]
    active = np.ones(r, dtype=bool)
    if f_target is not None:
        active &= f > f_target
    iters = np.zeros(r, dtype=int)
    calls = 1
    history = [float(np.min(f))]

    def direction(i):
        q = g[i].copy()
        alphas = []
        for s, y in zip(reversed(S[i]), reversed(Y[i])):
            rho = 1.0 / float(y @ s)
            a = rho * float(s @ q)
            alphas.append((a, rho, s, y))
            q -= a * y
        if S[i]:
            s, y = S[i][-1], Y[i][-1]
            q *= float(s @ y) / float(y @ y)
        for a, rho, s, y in reversed(alphas):
            b = rho * float(y @ q)
            q += (a - b) * s
        d = -q
        if float(d @ g[i]) >= 0:  # not a descent direction: restart from steepest descent
            S[i].clear()
            Y[i].clear()
            d = -g[i]
        return d

    dirs = np.zeros_like(x)
    steps = np.ones(r)
    backtracks = np.zeros(r, dtype=int)
    fresh = np.ones(r, dtype=bool)  # needs a new direction
    while active.any():
        idx = np.nonzero(active)[0]
        for i in idx:
            if fresh[i]:
                dirs[i] = direction(i)
                gnorm = float(np.linalg.norm(g[i]))
                steps[i] = 1.0 if S[i] else min(1.0, 0.1 / max(gnorm, 1e-300))
                if max_step is not None:
                    steps[i] = min(steps[i], max_step / max(float(np.linalg.norm(dirs[i])), 1e-300))
                backtracks[i] = 0
                fresh[i] = False
        trial = x[idx] + steps[idx, None] * dirs[idx]
        ft, gt = fg(trial)
        calls += 1
        for k, i in enumerate(idx):
            slope = float(dirs[i] @ g[i])
            if ft[k] <= f[i] + c1 * steps[i] * slope:
                s = trial[k] - x[i]
                y = gt[k] - g[i]
                if float(y @ s) > 1e-300:
                    S[i].append(s)
                    Y[i].append(y)
                    if len(S[i]) > memory:
                        S[i].pop(0)
                        Y[i].pop(0)
                decrease = f[i] - ft[k]
                x[i], f[i], g[i] = trial[k], ft[k], gt[k]
                iters[i] += 1
                fresh[i] = True
                if (f_target is not None and f[i] <= f_target) or iters[i] >= max_iter or decrease <= rel_tol * max(abs(f[i]), 1e-300):
                    active[i] = False
            else:
                steps[i] *= 0.5
                backtracks[i] += 1
                if backtracks[i] > max_backtracks:
                    active[i] = False
        history.append(float(np.min(f)))
        if callback:
            callback(calls, x, f)
    return x, f, {"iterations": iters, "evaluations": calls, "history": history}


def lbfgs_device(fg, x0, max_iter=30, memory=8, rel_target=None, c1=1e-4, max_backtracks=12, device="cuda", callback=None, max_step=None):
    """L-BFGS on many independent starting points at once with its state on the GPU: points, gradients, the curvature
    pairs of every restart (a ring of `memory` pairs each), the two-loop recursion and the Armijo backtracking are
    torch float64 tensors on `device`, computed for all restarts together. fg(X) takes and returns device tensors
    (X [R, P] -> f [R], g [R, P]) and is called on every row each time (rows that stopped keep their point), so the
    evaluator's batch keeps its size. A restart stops when f <= rel_target x its starting f, after max_iter accepted
    steps, or after max_backtracks halvings of one step. With max_step, a trial step is at most that long (as in
    lbfgs_batched). Returns (x, f, info) as tensors on the device; info holds the evaluation count and the best
    objective after each evaluation."""
    import torch

    x = torch.as_tensor(x0, dtype=torch.float64, device=device).clone()
    R, P = x.shape
    f, g = fg(x)
    f0 = f.clone()
    S = torch.zeros(R, memory, P, dtype=torch.float64, device=device)
    Y = torch.zeros_like(S)
    rho = torch.zeros(R, memory, dtype=torch.float64, device=device)
    count = torch.zeros(R, dtype=torch.long, device=device)
    head = torch.zeros(R, dtype=torch.long, device=device)
    active = torch.ones(R, dtype=torch.bool, device=device)
    if rel_target is not None:
        active &= f > rel_target * f0
    iters = torch.zeros(R, dtype=torch.long, device=device)
    backtracks = torch.zeros(R, dtype=torch.long, device=device)
    step = torch.ones(R, dtype=torch.float64, device=device)
    d = torch.zeros_like(x)
    fresh = torch.ones(R, dtype=torch.bool, device=device)
    rows = torch.arange(R, device=device)
    history = [float(f.min())]
    calls = 1

    def direction(gr):
        q = gr.clone()
        alphas = []
        for j in range(memory):
            idx = (head - 1 - j) % memory
            valid = (j < count).to(torch.float64)
            s_, y_, r_ = S[rows, idx], Y[rows, idx], rho[rows, idx]
            a = valid * r_ * (s_ * q).sum(1)
            q = q - a[:, None] * y_
            alphas.append((a, idx, valid))
        newest = (head - 1) % memory
        s_n, y_n = S[rows, newest], Y[rows, newest]
        gamma = torch.where(count > 0, (s_n * y_n).sum(1) / (y_n * y_n).sum(1).clamp_min(1e-300), torch.ones_like(f))
        q = q * gamma[:, None]
        for a, idx, valid in reversed(alphas):
            b = valid * rho[rows, idx] * (Y[rows, idx] * q).sum(1)
            q = q + (a - b)[:, None] * S[rows, idx]
        return -q

    while bool(active.any()):
        if bool(fresh.any()):
            nd = direction(g)
            descent = (nd * g).sum(1) < 0
            nd = torch.where(descent[:, None], nd, -g)
            count = torch.where(fresh & ~descent, torch.zeros_like(count), count)
            d = torch.where(fresh[:, None], nd, d)
            gnorm = g.norm(dim=1)
            first = torch.where(count > 0, torch.ones_like(step), torch.clamp(0.1 / gnorm.clamp_min(1e-300), max=1.0))
            if max_step is not None:
                first = torch.minimum(first, max_step / d.norm(dim=1).clamp_min(1e-300))
            step = torch.where(fresh, first, step)
            backtracks = torch.where(fresh, torch.zeros_like(backtracks), backtracks)
            fresh = torch.zeros_like(fresh)
        trial = torch.where(active[:, None], x + step[:, None] * d, x)
        ft, gt = fg(trial)
        calls += 1
        slope = (d * g).sum(1)
        ok = active & (ft <= f + c1 * step * slope)
        # accepted steps: store the curvature pair when it is positive
        s_new, y_new = trial - x, gt - g
        sy = (s_new * y_new).sum(1)
        keep = ok & (sy > 1e-300)
        S[rows[keep], head[keep]] = s_new[keep]
        Y[rows[keep], head[keep]] = y_new[keep]
        rho[rows[keep], head[keep]] = 1.0 / sy[keep]
        head = torch.where(keep, (head + 1) % memory, head)
        count = torch.where(keep, torch.clamp(count + 1, max=memory), count)
        x = torch.where(ok[:, None], trial, x)
        f = torch.where(ok, ft, f)
        g = torch.where(ok[:, None], gt, g)
        iters = iters + ok.long()
        fresh = ok.clone()
        failed = active & ~ok
        step = torch.where(failed, step * 0.5, step)
        backtracks = backtracks + failed.long()
        done = (iters >= max_iter) | (backtracks > max_backtracks)
        if rel_target is not None:
            done |= f <= rel_target * f0
        active &= ~done
        history.append(float(f.min()))
        if callback:
            callback(calls, x, f)
    return x, f, {"iterations": iters, "evaluations": calls, "history": history, "f0": f0}


def random_search(evaluator, objective, kinds=KIND_PARAMS, rounds=5, batch=264, span=0.3, shrink=0.5, seed=20261008, log=None):
    """The reference's batched search (tools/py/calibrate_gpu.py:96-125): each round one batch of log-uniform points
    around the current best (the origin, the compiled model's own values, first), keep the best, shrink the box.
    Points are drawn from random.Random(seed) in the reference's order. Returns (best J, best log scales, history)."""
    rng = random.Random(seed)
    centre = {k: 0.0 for k in kinds}
    best = (math.inf, None)
    history = []
    for rnd in range(rounds):
        points = [{k: 0.0 for k in kinds}] if rnd == 0 else []
        while len(points) < batch:
            points.append({k: centre[k] + rng.uniform(-span, span) for k in kinds})
        thetas = np.array([[p[k] for k in kinds] for p in points])
        t0 = time.time()
        scores = [objective(inst) for inst in evaluator.run(thetas)]
        order = sorted(range(len(points)), key=lambda i: scores[i])
        top = order[0]
        history.append({"round": rnd, "points": len(points), "seconds": time.time() - t0, "best": scores[top],
                        "scales": {k: math.exp(v) for k, v in points[top].items()}})
        if log:
            log(history[-1])
        if scores[top] < best[0]:
            best = (scores[top], dict(points[top]))
        centre = dict(points[top])
        span *= shrink
    return best[0], best[1], history


# ------------------------------------------------------------------------------------------ torch

def batch_loss(theta, evaluator, objective, h_rel=DEFAULT_FD_STEP):
    """Objective of every row of theta (a float64 torch tensor [R, P]) as a differentiable torch value.

    With an AdjointEvaluator the forward runs every point forward and back on the GPU (the hand-written adjoint) and the
    backward returns the adjoint gradients; with a BatchEvaluator the forward runs the points and their central-
    difference stencils in one batch and the backward returns those differences."""
    import torch

    class _BatchObjective(torch.autograd.Function):
        @staticmethod
        def forward(ctx, th):
            if isinstance(evaluator, AdjointEvaluator):
                f, g, _ = evaluator.value_and_grad(th.detach().cpu().numpy(), objective)
            else:
                f, g = value_and_grad(evaluator, objective, th.detach().cpu().numpy(), h_rel)
            ctx.save_for_backward(torch.as_tensor(g, dtype=th.dtype, device=th.device))
            return torch.as_tensor(f, dtype=th.dtype, device=th.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out[:, None] * g

    return _BatchObjective.apply(theta)


# ------------------------------------------------------------------------------------------ command line

def _model_paths(args):
    from .files import decompressed

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ship = args.ship or decompressed(os.path.join(here, "tests", "golden", "titanic64.ship.json.gz"))
    sim = args.sim or decompressed(os.path.join(here, "tests", "golden", "titanic.sim.json.gz"))
    return ship, sim


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sinksim_b200.calibrate")
    ap.add_argument("mode", choices=("search", "lbfgs"))
    ap.add_argument("--ship")
    ap.add_argument("--sim")
    ap.add_argument("--numerics", default="portable")
    ap.add_argument("--observations", help="observations file (search mode)")
    ap.add_argument("--rounds", type=int, default=5)
    ap.add_argument("--batch", type=int, default=264)
    ap.add_argument("--span", type=float, default=0.3)
    ap.add_argument("--shrink", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=20261008)
    ap.add_argument("--restarts", type=int, default=64)
    ap.add_argument("--iters", type=int, default=30)
    ap.add_argument("--h", type=float, default=DEFAULT_FD_STEP, help="relative central-difference step")
    ap.add_argument("--gradient", default="fd", choices=("fd", "adjoint"),
                    help="fd: central differences on the batched forward (L-BFGS in host numpy); adjoint: the engine's adjoint "
                         "with the L-BFGS state on the GPU (torch)")
    ap.add_argument("--max-step", type=float, default=0.3, help="longest L-BFGS trial step, in parameter units (0: no limit)")
    ap.add_argument("--rel-target", type=float, default=None, help="stop a restart once its objective falls below this fraction of its start")
    ap.add_argument("--t-end", type=float, default=7920.0, help="s: the last of the 8 objective times")
    ap.add_argument("--liner", action="store_true", help="the generated benchmark liner (hullgen) instead of titanic64")
    ap.add_argument("--space", default="kinds", choices=("kinds", "workload"),
                    help="kinds: log scales of breach/over/down/top; workload: the configurations' 10 parameters "
                         "(door/over/down/top log scales and the six open breaches' areas, points drawn as the configurations do)")
    args = ap.parse_args(argv)
    if args.liner:
        import tempfile

        from . import hullgen

        args.ship, args.sim = hullgen.write(os.path.join(tempfile.gettempdir(), "sinksim_b200_liner"))
    ship, sim = _model_paths(args)
    if args.mode == "search":
        if not args.observations:
            ap.error("search needs --observations")
        with open(args.observations) as f:
            obs = json.load(f)
        ob = obs["objective"]
        ev = BatchEvaluator(ship, sim, numerics=args.numerics, t_max=ob["tMaxMin"] * 60, curve_every=ob["historyEverySec"])
        J, p, _ = random_search(ev, lambda inst: oracle_objective(inst, obs), rounds=args.rounds, batch=args.batch, span=args.span,
                                shrink=args.shrink, seed=args.seed, log=lambda h: print(json.dumps(h)))
        print(json.dumps({"best": J, "scales": {k: math.exp(v) for k, v in p.items()}, "instances": ev.instances,
                          "device_s": ev.device_ms / 1e3}))
        return 0
    # lbfgs: hidden kind scales drawn from the seed, the target trajectory from them, restarts from lognormal draws
    # under torchrun (one process per GPU) every rank runs its block of each evaluation's stencil and the objective
    # values are all-gathered, so every rank iterates the same L-BFGS
    from .shard import Ranks

    ranks = Ranks(backend="nccl")
    times = default_times(args.t_end)
    rng = np.random.default_rng(args.seed)
    space = None
    if args.space == "workload":
        from .files import load_model

        space = workload_space(load_model(ship, sim)[1])
    ev = BatchEvaluator(ship, sim, space=space, numerics=args.numerics, t_max=times[-1], curve_every=times[1] - times[0], device=ranks.local)
    if args.space == "workload":
        # fresh hidden parameters (the stream's points beyond the gradient workload's) and starts from the same law
        hidden = workload_point(ev.space, 10_000 + args.seed % 1000)
        x0 = np.stack([workload_point(ev.space, 20_000 + k) for k in range(args.restarts)])
    else:
        hidden = rng.normal(0.0, 0.3, size=ev.space.dim)
        x0 = rng.normal(0.0, 0.3, size=(args.restarts, ev.space.dim))
    target = TrajectoryObjective.from_target(ev.run(hidden[None, :])[0], times)
    t0 = time.time()
    trace = []  # (wall s, best objective so far) after every evaluation

    def note(f):
        best_now = float(np.min(np.asarray(f)))
        trace.append((time.time() - t0, min(best_now, trace[-1][1]) if trace else best_now))

    if args.gradient == "adjoint":
        import torch

        adj = AdjointEvaluator(ship, sim, space=ev.space, t_max=times[-1], device=ranks.local)
        dev = torch.device("cuda", ranks.local)

        def fg(X):
            f, g, _ = adj.value_and_grad(X.cpu().numpy(), target)
            note(f)
            return torch.as_tensor(f, device=dev), torch.as_tensor(g, device=dev)

        xt, ft, info = lbfgs_device(fg, x0, max_iter=args.iters, rel_target=args.rel_target, device=dev, max_step=args.max_step or None)
        x, fx = xt.cpu().numpy(), ft.cpu().numpy()
        ev.device_ms += adj.device_ms
        ev.instances += adj.instances
    else:
        def fg_fd(X):
            f, g = value_and_grad(ev, target, X, args.h, ranks=ranks)
            note(f)
            return f, g

        x, fx, info = lbfgs_batched(fg_fd, x0, max_iter=args.iters, max_step=args.max_step or None)
    wall = ranks.max(time.time() - t0)
    device_s = ranks.max(ev.device_ms / 1e3)
    instances = ranks.sum(float(ev.instances))
    best = int(np.argmin(fx))
    if ranks.rank == 0:
        # the relative objective: the best objective over the best of the starting points'
        start = trace[0][1]
        reached = {}
        for level in (1e-2, 1e-4, 1e-6):
            hit = next((t for t, b in trace if b <= level * start), None)
            reached[f"{level:g}"] = hit
        print(json.dumps({"gradient": args.gradient, "restarts": args.restarts, "gpus": ranks.world, "space": args.space,
                          "t_end": args.t_end, "iters": args.iters, "max_step": args.max_step,
                          "best_objective": float(fx[best]), "start_objective": start, "relative_objective": float(fx[best]) / start,
                          "wall_s_to_relative": reached, "recovery_error": float(np.max(np.abs(x[best] - hidden))),
                          "hidden": [float(v) for v in hidden], "best_point": [float(v) for v in x[best]],
                          "evaluations": info["evaluations"], "instances": instances, "wall_s": wall, "device_s": device_s}))
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
