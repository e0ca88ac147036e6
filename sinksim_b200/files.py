"""Reading compiled ship and sim files into numpy arrays on the host (for workload generation and checks; the
engine itself parses and verifies the files in C++)."""
import gzip
import json
import os
import shutil
import tempfile

import numpy as np


def decompressed(path):
    """A plain-file path for `path`: itself, or its gzip content unpacked once into a temporary cache."""
    if not str(path).endswith(".gz"):
        return path
    cache = os.path.join(tempfile.gettempdir(), "sinksim_b200_fixtures")
    os.makedirs(cache, exist_ok=True)
    dst = os.path.join(cache, os.path.basename(path)[:-3])
    if not os.path.exists(dst) or os.path.getmtime(dst) < os.path.getmtime(path):
        tmp = f"{dst}.{os.getpid()}.tmp"
        with gzip.open(path, "rb") as f, open(tmp, "wb") as g:
            shutil.copyfileobj(f, g)
        os.replace(tmp, dst)
    return dst


def read_json(path):
    if str(path).endswith(".gz"):
        with gzip.open(path, "rt") as f:
            return json.load(f)
    with open(path) as f:
        return json.load(f)


def _f64(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64))


def _i32(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


def _u8(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.uint8))


def load_model(ship_path, sim_path):
    """The arrays of a compiled ship and sim (the members the kernel reads) as two dicts of numpy arrays."""
    s = read_json(ship_path)
    m = read_json(sim_path)
    c, n, g = s["columns"], s["nodes"], s["segments"]
    ship = dict(x=_f64(c["x"]), y=_f64(c["y"]), dxdy=_f64(c["dxdy"]), zlo=_f64(c["zlo"]), zhi=_f64(c["zhi"]),
                segCol=_i32(g["col"]), segA=_f64(g["a"]), segE=_f64(g["e"]), mu=_f64(n["mu"]), vmax=_f64(n["vmax"]),
                amin=_f64(n["amin"]), aov=_f64(n["aov"]), segStart=_i32(n["segStart"]), segCount=_i32(n["segCount"]))
    G, K, Mo, Mk, Fo, B, R, S0 = (m[k] for k in ("groups", "connections", "monitors", "marks", "founder", "body", "readout", "state0"))
    sim = dict(rho=float(m["constants"]["rho"]), g=float(m["constants"]["g"]), dt=float(m["scheme"]["dt"]),
               gStart=_i32(G["nodeStart"]), gCount=_i32(G["nodeCount"]), gNodes=_i32(G["nodes"]), gMode=_u8(G["mode"]),
               gpx=_f64(G["px"]), gpy=_f64(G["py"]), gpz=_f64(G["pz"]), gMargin=float(G["margin"]),
               ca=_i32(K["a"]), cb=_i32(K["b"]), law=_u8(K["type"]), cx=_f64(K["x"]), cy=_f64(K["y"]), cz=_f64(K["z"]),
               area=_f64(K["area"]), coef=_f64(K["coef"]), kind=_u8(K["kind"]), idx=_i32(K["idx"]), en=_u8(K["en"]),
               tOn=_f64(K["tOn"]), skipGroup=_i32(K["skipGroup"]), monitor=_i32(K["monitor"]),
               kindNames=list(K.get("kindNames", [])),
               nmon=len(Mo["id"]), monThreshold=float(Mo["threshold"]), monitorId=list(Mo["id"]), markId=list(Mk["id"]),
               mkx=_f64(Mk["x"]), mky=_f64(Mk["y"]), mkz=_f64(Mk["z"]), mkWhen=_u8(Mk["when"]),
               founder=[float(Fo[k]) for k in ("hullTopBelow", "pitchAbsAbove", "buoyancyBelow", "minT")],
               body=[float(B["ms"]), float(B["KG"]), *map(float, B["g0"]), float(B["XO"]), float(B["YO"]),
                     *(float(B[k]) for k in ("mh0", "Ith0", "Iph0", "cDz", "cDth", "cDph", "qz", "qth", "qph"))],
               xFP=float(R["xFP"]), xAP=float(R["xAP"]),
               state0=[float(S0[k]) for k in ("t", "zO", "pitch", "roll", "vz", "wth", "wph")],
               vol0=_f64(S0["vol"]), level0=_f64(S0["level"]), cx0=_f64(S0["cx"]), cy0=_f64(S0["cy"]), cz0=_f64(S0["cz"]))
    return ship, sim
