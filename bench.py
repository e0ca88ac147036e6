"""Benchmark of the batch time-stepper: aggregate sim-steps/s on B200s, bit-exact portable numerics.

Workload ("uneven run length" batch on the titanic64 model, the reference's compiled 4,408-column, 64-space,
290-connection hull): COUNT instances per GPU, each with its own connection-kind scale factors (lognormal(0, 0.3) on
breach/over/down/top), doors opened with probability 0.2, run until it founders, sinks (|trim| > 15 deg with the bow
deck edge under water), settles (|pitch rate| < 1e-5 rad/s for 600 s) or reaches tMax. One bench "step" is one
complete batch: every instance from its initial state to its end, in one persistent launch.

  value   total sim-steps of all ranks / the slowest rank's device time (CUDA events around the kernel launches on
          the engine's stream), inputs resident in HBM
  e2e     the same through the public API (Batch upload + launch + download: host inputs -> device, run, results ->
          host) timed on the host around each run
The CPU baseline is the reference CPU engine (oracle/_ref, built from the reference's own sources) on a seeded random
sample of whole runs of the same instances (founder, sink/settle rule or tMax, as on the GPU), all host cores;
--impl reference times that alone.

Other workloads: --workload fleet (a mixed fleet of generated hulls, one instance each, in one batch) and
--workload gradient (gradients/s of a 10-parameter trajectory objective on the generated liner by the hand-written
adjoint, one step = one public gradient call over the points; the finite-difference arm, 21 runs per gradient, and one
forward run of the same points are timed beside it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--numerics portable|portable32]
                    [--model titanic64|liner] [--workload uneven|fleet|gradient]
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic FP64 work of one titanic64 step (separately rounded adds, multiplies, divides, square roots; compares
# and min/max not counted), from the exact per-step unit counts of the C restatement over a full run
# (tests/test_oracle.py::test_work_counts_titanic64): 4,408 column clips (7 ops dry, 18 wet; 4,058 wet), 9,422
# segment visits (10 ops dry, 21.5 wet; 4,174 wet), 71 node-pass trees (31), the buoyancy tree (191), 27 weir pows
# (75), 290 connection flows (30), 64 node updates and loads (40).
FP64_OPS_PER_STEP = 7 * 4408 + 11 * 4058 + 10 * 9422 + 11.5 * 4174 + 71 * 31 + 191 + 75 * 27 + 30 * 290 + 40 * 64

# DRAM bytes (read + write) of one main-phase launch over the 4,096 instances, from ncu (dram__bytes per second x
# duration of run_batch<portable, 2-warp teams> on the same batch run to 600 s: python bench.py --count 4096 --tmax 600).
# The traffic is the instances' state going in and out: the geometry and the running state stay on chip, so the figure
# does not grow with the steps a launch takes.
KERNEL_DRAM_BYTES_PER_LAUNCH = 24.6e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--numerics", default="portable", choices=("portable", "portable32"))
    ap.add_argument("--count", type=int, default=None, help="instances per GPU (uneven: 4096, perturbed: 264)")
    ap.add_argument("--tmax", type=float, default=None, help="s (uneven: 5 h, perturbed: 2.6 h)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--model", default=None, choices=("titanic64", "liner"),
                    help="titanic64: the reference's compiled model; liner: the generated benchmark liner "
                         "(default: liner for --workload gradient, else titanic64)")
    ap.add_argument("--workload", default="uneven", choices=("uneven", "perturbed", "fleet", "gradient"),
                    help="uneven: one model, uneven run lengths; perturbed: the plain method's GPU form, seed-perturbed copies "
                         "of one model (the reference's --perturb: breach areas x (1 + 0.02 i / count)) run to founder or tmax; "
                         "fleet: a mixed fleet of generated hulls in one batch; gradient: gradients of a trajectory objective")
    ap.add_argument("--hulls", type=int, default=2048, help="fleet: hulls per GPU (one instance each)")
    ap.add_argument("--fleet-tmax", type=float, default=7200.0, help="fleet: s; instances also stop when they founder or calm down")
    ap.add_argument("--points", type=int, default=256, help="gradient: parameter points per GPU (one gradient each)")
    ap.add_argument("--fd-steps", type=int, default=1, help="gradient: timed calls of the finite-difference arm (0: none)")
    ap.add_argument("--t-end", type=float, default=7920.0, help="gradient: s, the last of the objective's 8 times and the runs' end")
    ap.add_argument("--tape-gb", type=float, default=0.0, help="gradient: device memory for the adjoint's step records (0: chosen)")
    ap.add_argument("--adjoint-warps", type=int, default=0, help="gradient: warps per adjoint team, 4, 8 or 16 (0: chosen)")
    ap.add_argument("--stage-columns", action="store_true", help="uneven: every block holds the column table in shared memory")
    ap.add_argument("--autotune", action="store_true", help="pick the launch shape by timing candidates first (outside the timed region)")
    args = ap.parse_args()
    if args.model is None:
        args.model = "liner" if args.workload in ("gradient", "perturbed") else "titanic64"
    if args.count is None:
        args.count = 264 if args.workload == "perturbed" else 4096
    if args.tmax is None:
        args.tmax = 2.6 * 3600.0 if args.workload == "perturbed" else 5 * 3600.0
    return args


def estimated_ops_per_step(columns, segments, nodes, connections):
    """FP64 operations of one step of a model, estimated from its sizes with titanic64's measured per-step ratios (92.1%
    of columns wet, 1.082 segment visits per segment with 44.3% of them wet, 1.109 node-pass trees per node, weir pows on
    9.3% of the connections) and the per-unit counts of FP64_OPS_PER_STEP; gives 233,388 for titanic64."""
    visits = 1.0822 * segments
    return (7 * columns + 11 * 0.9206 * columns + 10 * visits + 11.5 * 0.4430 * visits + 31 * 1.109 * nodes + 191
            + 75 * 0.0931 * connections + 30 * connections + 40 * nodes)


def _write_hull(job):
    """One generated fleet hull (run in a spawned worker): (index, seed, spec args, directory) -> (ship, sim) paths."""
    i, seed, spec, out = job
    from sinksim_b200 import hullgen

    return hullgen.write(out, spec=hullgen.HullSpec(**spec), seed=seed, ship_id=f"hull{i:05d}")


def fleet_models(count, first, seed=20261204):
    """The fleet's hulls first .. first+count-1, written in parallel; returns [(ship, sim)] and their sizes."""
    import multiprocessing

    from sinksim_b200 import hullgen

    specs = hullgen.fleet_specs(first + count, seed=seed)[first:]
    out = os.path.join(tempfile.gettempdir(), f"sinksim_b200_fleet_{seed}")
    jobs = [(first + k, seed + first + k, vars(sp), out) for k, sp in enumerate(specs)]
    with multiprocessing.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        paths = pool.map(_write_hull, jobs, chunksize=8)
    return paths


MODELS = {
    "titanic64": "titanic64 (4408 columns, 64 spaces, 290 connections; the reference's compiled model)",
    "liner": "liner269 (generated 269 x 28 m liner: 4408 columns, 64 spaces, 290 connections)",
}


def model_paths(model="titanic64"):
    from sinksim_b200.files import decompressed

    if model == "liner":
        from sinksim_b200 import hullgen

        return hullgen.write(os.path.join(tempfile.gettempdir(), "sinksim_b200_bench_liner"))
    golden = os.path.join(ROOT, "tests", "golden")
    return decompressed(os.path.join(golden, "titanic64.ship.json.gz")), decompressed(os.path.join(golden, "titanic.sim.json.gz"))


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def instance_params(sim, count, first, args, total=None):
    """(area {conn: area}, enabled {conn: 0/1}) of instances first .. first+count-1 of the workload: the uneven batch's
    draws, or for `perturbed` the reference's --perturb (apps/sinksim_cuda_run.cpp:126-135): every breach connection's
    compiled area x (1 + 0.02 i / total) for instance i of `total` (i >= 1), one product each."""
    from sinksim_b200.workloads import batch_uneven

    if args.workload != "perturbed":
        return batch_uneven(sim, count, first=first)
    total = total or count
    kinds = list(sim["kindNames"])
    breach = [int(c) for c in range(len(sim["kind"])) if "breach" in kinds and sim["kind"][c] == kinds.index("breach")]
    out = []
    for i in range(first, first + count):
        area = {} if i == 0 else {c: float(sim["area"][c]) * (1 + 0.02 * i / total) for c in breach}
        out.append((area, {}))
    return out


def workload_rule(ship, args):
    """The uneven batch's sink/settle retire rule; the perturbed copies stop at their founder or tmax only."""
    from sinksim_b200.workloads import deck_edge_rule

    return None if args.workload == "perturbed" else deck_edge_rule(ship)


def _tune_log(shape, ms, steps):
    print(f"autotune: {shape} {ms:.1f} ms ({steps} sim-steps)", file=sys.stderr)


def make_batch(ssb, ship_p, sim_p, sim, rule, count, first, args, device, total=None, **shape):
    shape.setdefault("stage_columns", getattr(args, "stage_columns", False))
    b = ssb.Batch(ship_p, sim_p, count=count, numerics=args.numerics, t_max=args.tmax, device=device, rule=rule, **shape)
    for i, (area, enabled) in enumerate(instance_params(sim, count, first, args, total)):
        for c, a in area.items():
            b.set_connection_area(i, c, a)
        for c, e in enabled.items():
            b.set_connection_enabled(i, c, e)
    return b


def cpu_fleet_rate(hulls, numerics, threads, t_max):
    """The reference CPU engine on the fleet's first `threads` hulls, one sinksim_sweep process per hull in parallel;
    returns (aggregate steps/s, steps, s, hulls): the steps of all processes over the longest of their own run times
    (each process times its run, without its start-up and model loading)."""
    tool = os.path.join(ROOT, "oracle", "_ref", "sinksim_sweep")
    sample = hulls[:threads]
    with tempfile.TemporaryDirectory() as d:
        procs = []
        for k, (ship_p, sim_p) in enumerate(sample):
            sw = {"format": "sinksim.sweep", "formatVersion": 1, "ship": "", "sim": "", "tMax": t_max, "every": 30, "stopWhenStable": True,
                  "instances": [{"id": f"hull{k}"}]}
            p = os.path.join(d, f"h{k}.sweep.json")
            with open(p, "w") as f:
                json.dump(sw, f)
            procs.append(subprocess.Popen([tool, ship_p, sim_p, p, "--numerics", numerics, "--threads", "1"], stdout=subprocess.PIPE,
                                          stderr=subprocess.STDOUT, text=True))
        outs = [pr.communicate()[0] for pr in procs]
    steps, longest = 0, 0.0
    for pr, o in zip(procs, outs):
        if pr.returncode != 0:
            raise RuntimeError(o)
        m = re.search(r"(\d+) steps in ([0-9.]+) s", o)
        steps += int(m.group(1))
        longest = max(longest, float(m.group(2)))
    return steps / longest, steps, longest, len(sample)


def _reference_sweep(ship_p, sim_p, sw, numerics, threads):
    """Runs the reference CPU engine's own sweep tool on the sweep document `sw`; returns (steps, s) as the tool reports
    them (its run time, without start-up and model loading)."""
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "sample.sweep.json")
        with open(p, "w") as f:
            json.dump(sw, f)
        tool = os.path.join(ROOT, "oracle", "_ref", "sinksim_sweep")
        r = subprocess.run([tool, ship_p, sim_p, p, "--numerics", numerics, "--threads", str(threads)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    m = re.search(r"(\d+) steps in ([0-9.]+) s \((\d+) steps/s aggregate\)", r.stdout)
    return int(m.group(1)), float(m.group(2))


def workload_sweep(sim, count, t_max, args):
    """The workload's instances 0 .. count-1 as a sweep document (each instance's areas and door overrides)."""
    sw = {"format": "sinksim.sweep", "formatVersion": 1, "ship": "", "sim": "", "tMax": t_max, "every": 30, "stopWhenStable": False,
          "instances": []}
    for i, (area, enabled) in enumerate(instance_params(sim, count, 0, args)):
        conns = [{"conn": c, "area": a} for c, a in area.items()] + [{"conn": c, "enabled": bool(e)} for c, e in enabled.items()]
        sw["instances"].append({"id": f"i{i}", "connections": conns})
    return sw


RUN_SAMPLE_SEED = 20261206


def cpu_whole_runs_rate(ship_p, sim_p, ship, sim, numerics, count, sample, t_max, threads, args):
    """The reference CPU engine (oracle/_ref/libsinksim_ref.so, Simulation::run) on a seeded random sample of whole runs
    of the GPU workload's `count` instances: each sampled instance from its initial state to its founder, the sink or
    settle rule or t_max, exactly as the GPU batch runs it, so both engines take the same mix of steps. Returns
    (steps/s, steps, s, sample indices)."""
    import ctypes as C

    import numpy as np

    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libsinksim_ref.so"))
    f = lib.ssref_time_sweep_runs
    f.restype = C.c_longlong
    f.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    lib.ssref_last_error.restype = C.c_char_p
    picks = np.sort(np.random.default_rng(RUN_SAMPLE_SEED).choice(count, size=min(sample, count), replace=False)).astype(np.int32)
    r = workload_rule(ship, args)
    rule = None if r is None else np.array([r["pitch"], r["x"], r["y"], r["z"], r["wth"], r["settle"]], dtype=np.float64)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "workload.sweep.json")
        with open(path, "w") as fh:
            json.dump(workload_sweep(sim, count, t_max, args), fh)
        secs = C.c_double()
        steps = f(ship_p.encode(), sim_p.encode(), path.encode(), numerics.encode(), picks.ctypes.data, picks.size, t_max,
                  None if rule is None else rule.ctypes.data, threads, C.byref(secs))
    if steps < 0:
        raise RuntimeError(lib.ssref_last_error().decode())
    return steps / secs.value, int(steps), secs.value, picks


# The gradient workload: gradients of a trajectory objective over 10 parameters, by the adjoint (one run forward and back
# per point) and, beside it, by central differences (2 P + 1 = 21 runs per point, every stencil in one batch).
from sinksim_b200.calibrate import workload_point as gradient_point  # noqa: E402
from sinksim_b200.calibrate import workload_space as gradient_space  # noqa: E402


def gradient_times(t_end=7920.0):
    """The objective's 8 times, evenly spaced to t_end (by default 990 s apart, to 2.2 h), and the curve interval
    that records exactly them."""
    from sinksim_b200.calibrate import default_times

    times = default_times(t_end)
    return times, times[1] - times[0]


def gradient_sweep(space, thetas, h_rel):
    """The sweep document of the central-difference stencils of the rows of `thetas` (2 P + 1 instances each, in
    fd_stencil's order): each instance sets the areas its point gives, to founder or the last objective time."""
    from sinksim_b200.calibrate import fd_stencil

    times, every = gradient_times()
    return {"format": "sinksim.sweep", "formatVersion": 1, "ship": "", "sim": "", "tMax": times[-1], "every": every,
            "stopWhenStable": False,
            "instances": [{"id": f"p{k}", "connections": [{"conn": c, "area": a} for c, a in space.areas(row).items()]}
                          for k, row in enumerate(fd_stencil(thetas, h_rel))]}


def cpu_gradient_rate(ship_p, sim_p, space, thetas, h_rel, numerics, threads):
    """The reference CPU engine's sweep tool on the central-difference stencils of the rows of `thetas`; returns
    (gradients/s, steps, s)."""
    steps, secs = _reference_sweep(ship_p, sim_p, gradient_sweep(space, thetas, h_rel), numerics, threads)
    return len(thetas) / secs, steps, secs


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ship_p, sim_p = model_paths(args.model)
    from sinksim_b200.files import load_model

    _, sim = load_model(ship_p, sim_p)
    threads = os.cpu_count() or 1
    if args.workload == "gradient":
        return reference_gradient_arm(args, ship_p, sim_p, sim, threads)
    if args.workload == "fleet":
        return reference_fleet_arm(args, threads)
    ship, _ = load_model(ship_p, sim_p)
    n = 8 * threads
    for _ in range(args.warmup):
        cpu_whole_runs_rate(ship_p, sim_p, ship, sim, args.numerics, args.count, n, args.tmax, threads, args)
    tot_steps, tot_s = 0, 0.0
    for _ in range(args.steps):
        _, s, secs, _ = cpu_whole_runs_rate(ship_p, sim_p, ship, sim, args.numerics, args.count, n, args.tmax, threads, args)
        tot_steps += s
        tot_s += secs
    v = tot_steps / tot_s
    ends = "its founder or" if args.workload == "perturbed" else "its founder, the sink or settle rule or"
    sample = (f"a seeded random sample of {n} of the {args.count} instances, each run whole (to {ends} "
              f"{args.tmax:.0f} s) by the reference engine's Simulation::run on {threads} threads; the same runs every step")
    print(json.dumps({"impl": "reference", "metric": "sim-steps/s", "value": v, "unit": "sim-steps/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.numerics == "portable" else "f32+f64",
                      "data": "synthetic", "config": workload_config(args),
                      "cpu_baseline": {"value": v, "unit": "sim-steps/s", "cores": threads, "kind": "reference", "sample": sample},
                      "e2e": {"value": v, "unit": "sim-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def reference_fleet_arm(args, threads):
    """--impl reference for the fleet: the reference engine's sweep tool on the fleet's first `threads` hulls, one
    process per hull in parallel."""
    hulls = fleet_models(threads, 0)
    tot_steps, tot_s = 0, 0.0
    for _ in range(args.steps):
        _, s, secs, n = cpu_fleet_rate(hulls, args.numerics, threads, args.fleet_tmax)
        tot_steps += s
        tot_s += secs
    v = tot_steps / tot_s
    sample = f"the fleet's first {threads} hulls, one reference sinksim_sweep process each, each to its founder, calm or {args.fleet_tmax:.0f} s"
    print(json.dumps({"impl": "reference", "metric": "sim-steps/s", "value": v, "unit": "sim-steps/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.numerics == "portable" else "f32+f64",
                      "data": "synthetic", "config": workload_config(args),
                      "cpu_baseline": {"value": v, "unit": "sim-steps/s", "cores": threads, "kind": "reference", "sample": sample},
                      "e2e": {"value": v, "unit": "sim-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def reference_gradient_arm(args, ship_p, sim_p, sim, threads):
    """--impl reference for the gradient workload: the reference CPU engine's sweep tool on the stencils of a sample of
    the points, all host threads; prints the reference line in gradients/s."""
    import numpy as np

    from sinksim_b200.calibrate import DEFAULT_FD_STEP

    space = gradient_space(sim)
    k = max(1, threads // 2)
    thetas = np.stack([gradient_point(space, i) for i in range(k)])
    for _ in range(args.warmup):
        cpu_gradient_rate(ship_p, sim_p, space, thetas, DEFAULT_FD_STEP, args.numerics, threads)
    tot_s = 0.0
    for _ in range(args.steps):
        _, _, secs = cpu_gradient_rate(ship_p, sim_p, space, thetas, DEFAULT_FD_STEP, args.numerics, threads)
        tot_s += secs
    v = k * args.steps / tot_s
    sample = (f"the stencils of the first {k} points ({k * (2 * space.dim + 1)} runs) per step, "
              f"reference sinksim_sweep --threads {threads}")
    print(json.dumps({"impl": "reference", "metric": "gradients/s", "value": v, "unit": "gradients/s", "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.numerics == "portable" else "f32+f64",
                      "data": "synthetic", "config": workload_config(args),
                      "cpu_baseline": {"value": v, "unit": "gradients/s", "cores": threads, "kind": "reference", "sample": sample},
                      "e2e": {"value": v, "unit": "gradients/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def workload_config(args):
    if args.workload == "gradient":
        return {"workload": f"gradients of a trajectory objective on {args.model}, {args.points} points per GPU, by the adjoint",
                "model": MODELS[args.model], "global_batch": args.points * args.gpus,
                "parameters": "10: log scale factors of the door, overflow, deck-opening and weather-deck-opening connections; "
                              "areas of the first 6 open breaches",
                "points": "kind scales lognormal(0, 0.3), breach areas U(0.1, 0.4) m2 (seeded); the target trajectory is the run at "
                          "a hidden point from the same distribution",
                "objective": f"sum of squared trim (deg) and heave (m) residuals at 8 times, evenly spaced to {args.t_end:g} s",
                "gradient": "hand-written FP64 discrete adjoint, one run forward (packed step records kept in HBM, checkpoints every "
                            "256 steps for what the records' memory does not hold) and back per gradient; "
                            "finite-difference arm beside it: central differences, relative step 1e-2, 21 runs per gradient",
                "numerics": args.numerics, "t_max_s": args.t_end, "dt_s": 0.25, "retire": "founder | tMax",
                "parallelism": f"points sharded over {args.gpus} GPU(s), no collective in the step",
                "l2": "working set (geometry 0.6 MB, per-instance state) is L2-resident by design; every step is a full batch from initial state"}
    if args.workload == "fleet":
        return {"workload": f"mixed fleet of {args.hulls} generated hulls per GPU, one instance each, in one batch",
                "model": "hulls of 1,000-20,000 columns (log-uniform, 5:1 grid), 16-256 spaces, 3-5 connections per space, L U(100, 300) m",
                "global_batch": args.hulls * args.gpus, "numerics": args.numerics, "t_max_s": args.fleet_tmax, "dt_s": 0.25,
                "retire": "founder | the reference's calm rule (stopWhenStable) | tMax",
                "parallelism": f"hulls sharded over {args.gpus} GPU(s), no collective in the step",
                "l2": "working set exceeds L2 for the largest hulls' geometry only; every step is a full batch from initial state"}
    if args.workload == "perturbed":
        return {"workload": f"{args.model}: {args.count} seed-perturbed copies per GPU (breach areas x (1 + 0.02 i / count), the "
                            f"reference's --perturb)", "model": MODELS[args.model], "global_batch": args.count * args.gpus,
                "numerics": args.numerics, "t_max_s": args.tmax, "dt_s": 0.25, "retire": "founder | tMax",
                "parallelism": f"instances sharded over {args.gpus} GPU(s), no collective in the step",
                "l2": "working set (geometry 0.6 MB, per-instance state) is L2-resident by design; every step is a full batch from initial state",
                "column_table": "shared memory of every block (bulk asynchronous copies)" if args.stage_columns else "global memory, through L1"}
    return {"workload": f"{args.model} uneven-run-length batch, {args.count} instances per GPU", "model": MODELS[args.model],
            "global_batch": args.count * args.gpus, "numerics": args.numerics, "t_max_s": args.tmax, "dt_s": 0.25,
            "retire": "founder | sink (|trim|>15 deg, bow deck edge under) | settle (|pitch rate|<1e-5 rad/s for 600 s) | tMax",
            "parallelism": f"instances sharded over {args.gpus} GPU(s), no collective in the step",
            "l2": "working set (geometry 0.6 MB, per-instance state) is L2-resident by design; every step is a full batch from initial state",
            "column_table": "shared memory of every block (bulk asynchronous copies)" if args.stage_columns else "global memory, through L1"}


def gradient_bench(args):
    """The gradient workload on the GPU. One step is one public gradient evaluation of the rank's points by the
    hand-written adjoint (AdjointEvaluator.value_and_grad: every point forward with FP64 checkpoints every 256 steps,
    then back); value from its kernel's CUDA-event time, e2e from its host time. Beside it: the same points' forward run
    alone (the adjoint's cost in forward runs) and the finite-difference arm (value_and_grad: 21 runs per gradient in one
    batch)."""
    import numpy as np

    import sinksim_b200 as ssb
    from sinksim_b200.calibrate import DEFAULT_FD_STEP, AdjointEvaluator, BatchEvaluator, TrajectoryObjective, value_and_grad
    from sinksim_b200.files import load_model
    from sinksim_b200.shard import Ranks, shard_bounds

    ranks = Ranks(backend="nccl", timeout_s=900)
    world, rank, local = ranks.world, ranks.rank, ranks.local
    ship_p, sim_p = model_paths(args.model)
    ship, sim = load_model(ship_p, sim_p)
    space = gradient_space(sim)
    times, every = gradient_times(args.t_end)
    ev = BatchEvaluator(ship_p, sim_p, space=space, numerics="portable", t_max=times[-1], curve_every=every, device=local)
    target = TrajectoryObjective.from_target(ev.run(gradient_point(space, -1)[None, :])[0], times)
    adj = AdjointEvaluator(ship_p, sim_p, space=space, t_max=times[-1], device=local, tape_budget=int(args.tape_gb * 2 ** 30),
                           team_warps=args.adjoint_warps)
    first, _ = shard_bounds(args.points * world, world, rank)
    thetas = np.stack([gradient_point(space, first + k) for k in range(args.points)])
    for _ in range(args.warmup):
        adj.value_and_grad(thetas, target)
    ranks.barrier()
    dev_ms, e2e_s, sim_steps = 0.0, 0.0, 0
    with Clocks(local) as clocks:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            f, g, steps = adj.value_and_grad(thetas, target)
            e2e_s += time.perf_counter() - t0
            dev_ms += adj.last["device_ms"]
            sim_steps += adj.last["steps"]
    ranks.barrier()
    if not (np.all(np.isfinite(f)) and np.all(np.isfinite(g))):
        raise RuntimeError("non-finite objective or gradient")
    # the same points' forward run alone (one batch, the objective's curves): one forward run's device time
    fwd_ms = []
    for k in range(2):
        ev.run(thetas)
        if k:
            fwd_ms.append(ev.last["device_ms"])
    # the finite-difference arm: every point's 21 runs in one batch
    fd_ms, fd_s = 0.0, 0.0
    if args.fd_steps:
        value_and_grad(ev, target, thetas, DEFAULT_FD_STEP)
    for _ in range(args.fd_steps):
        t0 = time.perf_counter()
        value_and_grad(ev, target, thetas, DEFAULT_FD_STEP)
        fd_s += time.perf_counter() - t0
        fd_ms += ev.last["device_ms"]
    dev_s_max = ranks.max(dev_ms / 1e3)
    e2e_max = ranks.max(e2e_s)
    fd_dev_max = ranks.max(fd_ms / 1e3) if args.fd_steps else None
    fd_e2e_max = ranks.max(fd_s) if args.fd_steps else None
    recomputed = ranks.sum(float(adj.last["recomputed"]))
    fwd_max = ranks.max(min(fwd_ms) / 1e3)
    grads = ranks.sum(float(args.points * args.steps))
    fd_grads = ranks.sum(float(args.points * args.fd_steps))
    all_steps = ranks.sum(float(sim_steps))
    clk = clocks.summary()
    if rank == 0:
        info = adj.last["info"]
        fp64_peak = ssb.add_mul_peak(True, local)
        if args.model == "titanic64":
            ops_per_step, ops_source = FP64_OPS_PER_STEP, "exact unit counts of titanic64 (the C restatement's counters)"
        else:
            ops_per_step = estimated_ops_per_step(len(ship["x"]), len(ship["segCol"]), len(ship["segCount"]), len(sim["ca"]))
            ops_source = "estimated from the model's size with titanic64's per-step ratios"
        adjoint_s = dev_s_max / args.steps
        # the kernel steps every run forward (recording every step), reverses every step and recomputes the steps its
        # ring of records no longer holds; the reverse of a step sweeps the same geometry as its forward (the node
        # passes' and columns' reverses), so each counts as one step's FP64 work
        step_equivalents = 2 * all_steps / args.steps + recomputed
        achieved = ops_per_step * step_equivalents / adjoint_s
        n_params = space.dim
        out = {"metric": "gradients/s", "value": grads / dev_s_max, "unit": "gradients/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": dev_s_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(args),
               "e2e": {"value": grads / e2e_max, "unit": "gradients/s", "h2d_bytes_per_step": info["h2d_bytes"],
                       "d2h_bytes_per_step": info["d2h_bytes"]},
               "gpu_launches": args.steps, "adjoint": {"team_warps": info["team_warps"], "teams": info["teams"], "checkpoint_every": 256,
                                                      "device_s_per_call": adjoint_s, "forward_run_s": fwd_max,
                                                      "cost_in_forward_runs": adjoint_s / fwd_max,
                                                      "sim_steps_per_run": all_steps / args.steps, "recomputed_steps": recomputed,
                                                      "ring_mb_per_team": adj.last["ring_bytes"] / 2 ** 20,
                                                      "team_s": dict(zip(("forward", "recompute", "reverse"), adj.last["phase_team_s"]))},
               "finite_difference_arm": None if not args.fd_steps else {
                   "value": fd_grads / fd_dev_max, "unit": "gradients/s", "e2e": fd_grads / fd_e2e_max,
                   "runs_per_gradient": 2 * n_params + 1, "relative_step": DEFAULT_FD_STEP, "calls": args.fd_steps},
               "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": fp64_peak / 1e12, "unit": "TFLOP/s",
                            "frac": achieved / fp64_peak, "traffic": None, "ops_source": ops_source,
                            "kernel": f"adjoint_batch<{info['team_warps']}-warp teams>",
                            "work": f"{step_equivalents:.0f} step-equivalents per call (forward and reverse of every sim-step, "
                                    f"plus {recomputed:.0f} recomputed)",
                            "peak_source": "measured on this GPU: separately rounded FP64 add+mul microbenchmark (no FMA, as the bits require)",
                            "ops_per_sim_step": ops_per_step},
               "clocks": clk}
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            k = max(1, threads // 2)
            v, s, secs = cpu_gradient_rate(ship_p, sim_p, space, thetas[:k], DEFAULT_FD_STEP, "portable", threads)
            out["cpu_baseline"] = {"value": v, "unit": "gradients/s", "cores": threads, "kind": "reference",
                                   "sample": f"central differences (21 runs each) at the first {k} points ({s} steps in {secs:.1f} s), "
                                             f"reference sinksim_sweep --numerics portable --threads {threads}"}
        print(json.dumps(out))
    adj.close()
    ranks.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "gradient":
        return gradient_bench(args)
    import numpy as np

    import sinksim_b200 as ssb
    from sinksim_b200.files import load_model
    from sinksim_b200.shard import Ranks, shard_bounds

    # one process per GPU; each rank steps its own contiguous block of the instances (weak scaling: count per GPU)
    ranks = Ranks(backend="nccl", timeout_s=600)
    world, rank, local = ranks.world, ranks.rank, ranks.local
    barrier, max_over_ranks, sum_over_ranks = ranks.barrier, ranks.max, ranks.sum
    shape, tune_table = {}, []
    if args.workload == "fleet":
        first, _ = shard_bounds(args.hulls * world, world, rank)
        hulls = fleet_models(args.hulls, first)

        def make_fleet(**s):
            return ssb.Batch.fleet(hulls, list(range(len(hulls))), numerics=args.numerics, t_max=args.fleet_tmax, device=local,
                                   stop_when_stable=True, **s)

        if args.autotune:
            from sinksim_b200.autotune import DEFAULT_SPACE, search

            # a fleet's slot is set by its largest hull and the column table is per model: no staged table
            shape, tune_table = search(make_fleet, space=tuple(d for d in DEFAULT_SPACE if d[0] != "stage_columns"), log=_tune_log)
        batch = make_fleet(**shape)
        hull_ops = []
        for ship_p, sim_p in hulls:
            s_doc, m_doc = load_model(ship_p, sim_p)
            hull_ops.append(estimated_ops_per_step(len(s_doc["x"]), len(s_doc["segCol"]), len(s_doc["segCount"]), len(m_doc["ca"])))
        ship_p, sim_p = hulls[0]
    else:
        ship_p, sim_p = model_paths(args.model)
        ship, sim = load_model(ship_p, sim_p)
        rule = workload_rule(ship, args)
        first, _ = shard_bounds(args.count * world, world, rank)
        total = args.count * world
        if args.autotune:
            from sinksim_b200.autotune import search

            shape, tune_table = search(lambda **s: make_batch(ssb, ship_p, sim_p, sim, rule, args.count, first, args, local, total, **s),
                                       log=_tune_log)
        batch = make_batch(ssb, ship_p, sim_p, sim, rule, args.count, first, args, local, total, **shape)
    # warm-up: full batches, untimed
    for _ in range(args.warmup):
        batch.reset()
        batch.run()
    # device-timed steps (value): inputs staged to HBM before each launch, the launch timed with CUDA events
    barrier()
    # each timed step is one public run (inputs host -> device, every instance to its end, results device -> host):
    # its wall time is the end-to-end figure, the CUDA-event time of its kernel launch the device figure
    dev_ms, steps_total, e2e_s = 0.0, 0, 0.0
    per_launch_ms = []
    phase_ms, phase_steps = None, None
    with Clocks(local) as clocks:
        for _ in range(args.steps):
            batch.reset()
            t0 = time.perf_counter()
            batch.upload()
            ms = batch.launch()
            batch.download()
            e2e_s += time.perf_counter() - t0
            dev_ms += ms
            per_launch_ms.append(ms)
            steps_total += batch.total_steps()
            ps = batch.phase_stats()
            phase_ms = [p["device_ms"] for p in ps] if phase_ms is None else [a + p["device_ms"] for a, p in zip(phase_ms, ps)]
            phase_steps = [p["steps"] for p in ps] if phase_steps is None else [a + p["steps"] for a, p in zip(phase_steps, ps)]
    barrier()
    h2d, d2h = batch.transfer_bytes()
    info = batch.launch_info()
    dev_s_max = max_over_ranks(dev_ms / 1e3)
    e2e_max = max_over_ranks(e2e_s)
    all_steps = sum_over_ranks(float(steps_total))
    clk = clocks.summary()
    if rank == 0:
        value = all_steps / dev_s_max
        e2e = all_steps / e2e_max
        fp64_peak = ssb.add_mul_peak(True, local)
        fp32_peak = ssb.add_mul_peak(False, local)
        steps_per_launch = steps_total / args.steps
        # the dominant kernel: the launch phase with the most device time; its work over its own CUDA-event time
        top = max(range(len(phase_ms)), key=lambda k: phase_ms[k])
        top_warps = batch.phase_stats()[top]["team_warps"]
        ops_per_step, ops_source = FP64_OPS_PER_STEP, "exact unit counts of titanic64 (the C restatement's counters)"
        traffic = KERNEL_DRAM_BYTES_PER_LAUNCH
        if args.workload == "fleet":  # the steps' mix of hulls: ops per step weighted by each instance's steps
            steps_i = [batch.summary(i)["steps"] for i in range(len(hull_ops))]
            ops_per_step = sum(o * s for o, s in zip(hull_ops, steps_i)) / max(sum(steps_i), 1)
            ops_source, traffic = "estimated from each hull's size with titanic64's per-step ratios", None
        elif args.model != "titanic64":
            ops_per_step = estimated_ops_per_step(len(ship["x"]), len(ship["segCol"]), len(ship["segCount"]), len(sim["ca"]))
            ops_source, traffic = "estimated from the model's size with titanic64's per-step ratios", None
        achieved = ops_per_step * phase_steps[top] / (phase_ms[top] / 1e3)
        phases = [{"team_warps": p["team_warps"], "device_ms_per_run": m / args.steps, "share": m / sum(phase_ms),
                   "sim_steps_per_run": s / args.steps} for p, m, s in zip(batch.phase_stats(), phase_ms, phase_steps)]
        out = {"metric": "sim-steps/s", "value": value, "unit": "sim-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": dev_s_max * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f64" if args.numerics == "portable" else "f32+f64", "data": "synthetic", "config": workload_config(args),
               "e2e": {"value": e2e, "unit": "sim-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "gpu_launches": args.steps * info["kernels"], "launch": info, "sim_steps_per_launch": steps_per_launch,
               "autotuned_shape": shape if args.autotune else None,
               "autotune_table": [[t[0], t[1]] for t in tune_table] if args.autotune else None,
               "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": fp64_peak / 1e12, "unit": "TFLOP/s",
                            "frac": achieved / fp64_peak, "traffic": traffic, "ops_source": ops_source,
                            "kernel": f"run_batch<{args.numerics}, {top_warps}-warp teams> (launch phase {top})",
                            "phases": phases,
                            "peak_source": "measured on this GPU: separately rounded FP64 add+mul microbenchmark (no FMA, as the bits require)",
                            "fp32_peak": fp32_peak / 1e12, "ops_per_sim_step": ops_per_step,
                            "note": "the step is issue/latency bound; HBM traffic is negligible (L2-resident working set)"},
               "clocks": clk}
        if world == 1 and not args.no_cpu_baseline and args.workload == "fleet":
            threads = os.cpu_count() or 1
            v, s, secs, n = cpu_fleet_rate(hulls, args.numerics, threads, 1800.0)
            out["cpu_baseline"] = {"value": v, "unit": "sim-steps/s", "cores": threads, "kind": "reference",
                                   "sample": f"the first {n} hulls of the fleet, one reference sinksim_sweep process each (in parallel), each to its "
                                             f"founder or 1800 s ({s} steps in {secs:.1f} s)"}
        elif world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            n = 8 * threads
            v, s, secs, _ = cpu_whole_runs_rate(ship_p, sim_p, ship, sim, args.numerics, args.count, n, args.tmax, threads, args)
            out["cpu_baseline"] = {"value": v, "unit": "sim-steps/s", "cores": threads, "kind": "reference",
                                   "sample": f"a seeded random sample of {n} of the {args.count} instances, each run whole ("
                                             f"{'founder' if args.workload == 'perturbed' else 'founder, sink or settle rule'}, "
                                             f"{args.tmax:.0f} s) by the reference engine on {threads} threads "
                                             f"({s} steps in {secs:.1f} s): the same step mix as the GPU batch"}
        print(json.dumps(out))
    batch.close()
    ranks.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
