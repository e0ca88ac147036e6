"""Writes the committed parity fixtures of this directory from the reference repository's own data files.

Run in a container that has the reference tree mounted (the GPU box does not need it):
    python tests/golden/make_fixtures.py [/path/to/reference]

It copies, gzip-compressed and unchanged in content:
  * ships/titanic/titanic64.ship.json and ships/titanic/sims/titanic.sim.json (the compiled titanic64 model that
    the reference's golden and GPU tests run, tests/CMakeLists.txt:11-65)
  * tests/sweeps/smoke.sweep.json (the reference's GPU-vs-CPU sweep fixture, tests/CMakeLists.txt:36-65)
and reduces the portable and portable32 golden traces (data/golden/titanic64/titanic.portable*.trace.json, held at
tolerance 0 by tests/CMakeLists.txt:19-28) to their first DENSE dense records and every sampled record. Values
are written with Python's shortest round-trip float repr, so every double survives exactly; the per-array hashes
are dropped because the arrays are shortened.
"""
import gzip
import json
import os
import shutil
import sys

DENSE = 60
HERE = os.path.dirname(os.path.abspath(__file__))
PER_NODE = ("vol", "level", "cx", "cy", "cz")


def reduce_trace(src, dst, dense):
    with open(src) as f:
        tr = json.load(f)
    nodes = tr["nodes"]
    d = tr["dense"]
    n = min(dense, d["n"])
    out = {}
    for k, v in d.items():
        if k == "n":
            out[k] = n
        elif k in PER_NODE:
            out[k] = v[: n * nodes]
        else:
            out[k] = v[:n]
    tr["dense"] = out
    tr.pop("hash", None)
    tr["role"] = "golden-reduced"
    with gzip.open(dst, "wt") as f:
        json.dump(tr, f, separators=(",", ":"))


def copy_gz(src, dst):
    with open(src, "rb") as f, gzip.open(dst, "wb") as g:
        shutil.copyfileobj(f, g)


def main(ref):
    copy_gz(os.path.join(ref, "ships/titanic/titanic64.ship.json"), os.path.join(HERE, "titanic64.ship.json.gz"))
    copy_gz(os.path.join(ref, "ships/titanic/sims/titanic.sim.json"), os.path.join(HERE, "titanic.sim.json.gz"))
    shutil.copyfile(os.path.join(ref, "tests/sweeps/smoke.sweep.json"), os.path.join(HERE, "smoke.sweep.json"))
    for tag in ("portable", "portable32"):
        reduce_trace(os.path.join(ref, f"data/golden/titanic64/titanic.{tag}.trace.json"),
                     os.path.join(HERE, f"titanic.{tag}.golden.json.gz"), DENSE)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SINKSIM_REFERENCE")
    if not ref:
        sys.exit("usage: make_fixtures.py <reference source tree> (or set SINKSIM_REFERENCE)")
    main(ref)
