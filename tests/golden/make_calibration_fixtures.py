"""Writes the calibration fixtures of this directory from the reference repository and its CPU engine.

Run in a container that has the reference tree mounted and oracle/_ref built (the GPU box does not need either):
    python tests/golden/make_calibration_fixtures.py [/path/to/reference]

  * titanic-1912.observations.json: the reference's data/observations/titanic-1912.json, unchanged (the observed
    trim, list, founder time and events and the objective's weights that tools/py/calibrate_gpu.py scores against).
  * calibration.points.json: six kind-scale points (the origin, then round 0 of the reference's random search:
    random.Random(20261008), log scales uniform in +-0.3 for breach, over, down, top, as calibrate_gpu.py:96-108
    draws them), the reference CPU engine's results for them (oracle/_ref/sinksim_sweep --numerics portable, tMax
    260 min, curves every 30 s), scored by the reference's own objective (calibrate_gpu.py:35-64, imported from the
    reference tree): J per point. The first two points' results are kept whole (calibration.results.json.gz) so the
    objective restatement can be checked on the CPU without the engine.
"""
import gzip
import json
import math
import os
import random
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
KINDS = ["breach", "over", "down", "top"]
SEED = 20261008
POINTS = 6


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SINKSIM_REFERENCE")
    if not ref:
        sys.exit("usage: make_calibration_fixtures.py <reference source tree> (or set SINKSIM_REFERENCE)")
    sys.path.insert(0, os.path.join(ref, "tools", "py"))
    import calibrate_gpu  # the reference's objective, used here only to score the fixture

    obs_src = os.path.join(ref, "data", "observations", "titanic-1912.json")
    shutil.copyfile(obs_src, os.path.join(HERE, "titanic-1912.observations.json"))
    with open(obs_src) as f:
        obs = json.load(f)
    ob = obs["objective"]
    rng = random.Random(SEED)
    points = [{k: 0.0 for k in KINDS}]
    while len(points) < POINTS:
        points.append({k: 0.0 + rng.uniform(-0.3, 0.3) for k in KINDS})
    sweep = {"format": "sinksim.sweep", "formatVersion": 1, "ship": "titanic64.ship.json", "sim": "titanic.sim.json",
             "tMax": ob["tMaxMin"] * 60, "every": ob["historyEverySec"], "stopWhenStable": False,
             "instances": [{"id": f"p{i}", "scale": {k: math.exp(v) for k, v in p.items()}} for i, p in enumerate(points)]}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _support import ref_tool, titanic

    ship_p, sim_p = titanic()
    with tempfile.TemporaryDirectory() as tmp:
        sw_p = os.path.join(tmp, "sweep.json")
        res_p = os.path.join(tmp, "results.json")
        with open(sw_p, "w") as f:
            json.dump(sweep, f)
        subprocess.run([ref_tool("sinksim_sweep"), ship_p, sim_p, sw_p, "--numerics", "portable", "--results", res_p], check=True)
        with open(res_p) as f:
            res = json.load(f)
    J = [calibrate_gpu.objective(inst, obs)[0] for inst in res["instances"]]
    with open(os.path.join(HERE, "calibration.points.json"), "w") as f:
        json.dump({"seed": SEED, "kinds": KINDS, "tMax": sweep["tMax"], "every": sweep["every"], "points": points,
                   "scales": [inst["scale"] for inst in sweep["instances"]], "J": J,
                   "steps": [inst["steps"] for inst in res["instances"]]}, f, indent=1)
    kept = dict(res, instances=res["instances"][:2])
    with gzip.open(os.path.join(HERE, "calibration.results.json.gz"), "wt") as f:
        json.dump(kept, f)
    print("J", J)


if __name__ == "__main__":
    main()
