"""Test helpers: fixtures, the compiled-model arrays, and ctypes wrappers over the checkers in oracle/_ref.

Only tests, __graft_entry__.smoke() and bench.py's CPU baseline use this module; the oracle is the checker of the
CUDA path, never part of it.
"""
import ctypes as C
import gzip
import json
import os
import shutil
import tempfile

import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
_CACHE = os.path.join(tempfile.gettempdir(), "sinksim_b200_fixtures")


def fixture(name):
    """Path of a fixture in tests/golden, decompressed into a temporary cache when it is stored gzip-compressed."""
    src = os.path.join(GOLDEN, name)
    if os.path.exists(src):
        return src
    gz = src + ".gz"
    if not os.path.exists(gz):
        raise FileNotFoundError(src)
    os.makedirs(_CACHE, exist_ok=True)
    dst = os.path.join(_CACHE, name)
    if not os.path.exists(dst) or os.path.getmtime(dst) < os.path.getmtime(gz):
        with gzip.open(gz, "rb") as f, open(dst + ".tmp", "wb") as g:
            shutil.copyfileobj(f, g)
        os.replace(dst + ".tmp", dst)
    return dst


from sinksim_b200.files import load_model, read_json  # noqa: E402,F401


def titanic():
    return fixture("titanic64.ship.json"), fixture("titanic.sim.json")


def f64(v):
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64))


def trace_records(tr, which):
    """Records of a trace's dense or samples block as an (n, 10 + 5 N) array in the record layout."""
    d = tr[which]
    N = tr["nodes"]
    n = d["n"]
    out = np.empty((n, 10 + 5 * N))
    for j, k in enumerate(("t", "zO", "pitch", "roll", "vz", "wth", "wph", "inflow", "Vb", "hullTop")):
        out[:, j] = d[k]
    for j, k in enumerate(("vol", "level", "cx", "cy", "cz")):
        out[:, 10 + j * N:10 + (j + 1) * N] = np.asarray(d[k], dtype=np.float64).reshape(n, N)
    return out


# ----------------------------------------------------------------------------------------------- the C restatement

def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class _Ship(C.Structure):
    _fields_ = [("ncol", C.c_int32), ("nseg", C.c_int32), ("nnode", C.c_int32)] + \
               [(k, C.POINTER(C.c_double)) for k in ("x", "y", "dxdy", "zlo", "zhi")] + \
               [("segCol", C.POINTER(C.c_int32))] + [(k, C.POINTER(C.c_double)) for k in ("segA", "segE", "mu", "vmax", "amin", "aov")] + \
               [(k, C.POINTER(C.c_int32)) for k in ("segStart", "segCount")]


class _Sim(C.Structure):
    _fields_ = [("rho", C.c_double), ("g", C.c_double), ("dt", C.c_double), ("ngroup", C.c_int32)] + \
               [(k, C.POINTER(C.c_int32)) for k in ("gStart", "gCount", "gNodes")] + [("gMode", C.POINTER(C.c_uint8))] + \
               [(k, C.POINTER(C.c_double)) for k in ("gpx", "gpy", "gpz")] + [("gMargin", C.c_double), ("nconn", C.c_int32)] + \
               [(k, C.POINTER(C.c_int32)) for k in ("ca", "cb")] + [("law", C.POINTER(C.c_uint8))] + \
               [(k, C.POINTER(C.c_double)) for k in ("cx", "cy", "cz", "area", "coef")] + [("en", C.POINTER(C.c_uint8)), ("tOn", C.POINTER(C.c_double))] + \
               [(k, C.POINTER(C.c_int32)) for k in ("skipGroup", "monitor")] + [("nmon", C.c_int32), ("monThreshold", C.c_double), ("nmark", C.c_int32)] + \
               [(k, C.POINTER(C.c_double)) for k in ("mkx", "mky", "mkz")] + [("mkWhen", C.POINTER(C.c_uint8))] + \
               [(k, C.c_double) for k in ("hullTopBelow", "pitchAbsAbove", "buoyancyBelow", "minT")] + \
               [("body", C.c_double * 16), ("xFP", C.c_double), ("xAP", C.c_double), ("state0", C.c_double * 7)] + \
               [(k, C.POINTER(C.c_double)) for k in ("vol0", "level0", "cx0", "cy0", "cz0")]


class _Counters(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("steps", "columns", "passes", "segVisits", "segWet", "colWet", "weirPow", "orifice", "weir", "newton")]


_oracle_lib = None


def oracle_lib():
    global _oracle_lib
    if _oracle_lib is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libsinksim_oracle.so"))
        lib.sso_create.restype = C.c_void_p
        lib.sso_create.argtypes = [C.POINTER(_Ship), C.POINTER(_Sim), C.c_int]
        for name in ("sso_destroy", "sso_reset"):
            getattr(lib, name).argtypes = [C.c_void_p]
        lib.sso_set_connection.argtypes = [C.c_void_p, C.c_int32, C.c_int, C.c_double, C.c_double]
        lib.sso_step.argtypes = [C.c_void_p, C.c_int64]
        lib.sso_get_record.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.sso_restore.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.sso_readouts.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.sso_events.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        lib.sso_foundered.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.sso_counters_get.argtypes = [C.c_void_p, C.POINTER(_Counters)]
        lib.sso_flows.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.sso_digest_start.argtypes = [C.c_void_p]
        lib.sso_digest.argtypes = [C.c_void_p]
        lib.sso_digest.restype = C.c_uint64
        _oracle_lib = lib
    return _oracle_lib


def _structs(ship, sim):
    """The oracle's C structs over a compiled model's arrays (the oracles copy them when they are created)."""
    S = _Ship(len(ship["x"]), len(ship["segCol"]), len(ship["mu"]),
              *(_p(ship[k], C.c_double) for k in ("x", "y", "dxdy", "zlo", "zhi")), _p(ship["segCol"], C.c_int32),
              *(_p(ship[k], C.c_double) for k in ("segA", "segE", "mu", "vmax", "amin", "aov")),
              _p(ship["segStart"], C.c_int32), _p(ship["segCount"], C.c_int32))
    m = sim
    M = _Sim(m["rho"], m["g"], m["dt"], len(m["gCount"]), _p(m["gStart"], C.c_int32), _p(m["gCount"], C.c_int32),
             _p(m["gNodes"], C.c_int32), _p(m["gMode"], C.c_uint8), _p(m["gpx"], C.c_double), _p(m["gpy"], C.c_double),
             _p(m["gpz"], C.c_double), m["gMargin"], len(m["ca"]), _p(m["ca"], C.c_int32), _p(m["cb"], C.c_int32),
             _p(m["law"], C.c_uint8), *(_p(m[k], C.c_double) for k in ("cx", "cy", "cz", "area", "coef")),
             _p(m["en"], C.c_uint8), _p(m["tOn"], C.c_double), _p(m["skipGroup"], C.c_int32), _p(m["monitor"], C.c_int32),
             m["nmon"], m["monThreshold"], len(m["mkx"]), *(_p(m[k], C.c_double) for k in ("mkx", "mky", "mkz")),
             _p(m["mkWhen"], C.c_uint8), *m["founder"], (C.c_double * 16)(*m["body"]), m["xFP"], m["xAP"],
             (C.c_double * 7)(*m["state0"]), *(_p(m[k], C.c_double) for k in ("vol0", "level0", "cx0", "cy0", "cz0")))
    return S, M


class Oracle:
    """The C restatement of the reference step (oracle/sinksim_oracle.c) on one compiled model."""

    def __init__(self, ship, sim, mixed=False):
        self.lib = oracle_lib()
        self.ship, self.sim = ship, sim
        self.nodes = len(ship["mu"])
        self.nconn = len(sim["ca"])
        S, M = _structs(ship, sim)
        self.h = self.lib.sso_create(C.byref(S), C.byref(M), 1 if mixed else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.sso_destroy(self.h)
            self.h = None

    def reset(self):
        self.lib.sso_reset(self.h)

    def set_connection(self, c, enabled=-1, area=float("nan"), tOn=float("nan")):
        self.lib.sso_set_connection(self.h, c, enabled, area, tOn)

    def step(self, n=1):
        self.lib.sso_step(self.h, n)

    def record(self):
        r = np.empty(10 + 5 * self.nodes)
        self.lib.sso_get_record(self.h, _p(r, C.c_double))
        return r

    def restore(self, rec):
        rec = f64(rec)
        self.lib.sso_restore(self.h, _p(rec, C.c_double))

    def readouts(self):
        r = np.empty(7)
        self.lib.sso_readouts(self.h, _p(r, C.c_double))
        return r

    def events(self):
        buf = np.empty(3 * 1024)
        n = self.lib.sso_events(self.h, _p(buf, C.c_double), 1024)
        return [(buf[3 * i], int(buf[3 * i + 1]), int(buf[3 * i + 2])) for i in range(n)]

    def foundered(self):
        t = C.c_double()
        f = self.lib.sso_foundered(self.h, C.byref(t))
        return bool(f), t.value

    def counters(self):
        c = _Counters()
        self.lib.sso_counters_get(self.h, C.byref(c))
        return {k: getattr(c, k) for k, _ in _Counters._fields_}

    def digest_start(self):
        self.lib.sso_digest_start(self.h)

    def digest(self):
        return int(self.lib.sso_digest(self.h))

    def flows(self):
        q = np.empty(self.nconn)
        self.lib.sso_flows(self.h, _p(q, C.c_double))
        return q


# ----------------------------------------------------------------------------------------------- the tangent-linear step

_tangent_lib = None
TANGENT_PARAMS = 10


def tangent_lib():
    global _tangent_lib
    if _tangent_lib is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libsinksim_tangent.so"))
        lib.sst_create.restype = C.c_void_p
        lib.sst_create.argtypes = [C.POINTER(_Ship), C.POINTER(_Sim)]
        lib.sst_destroy.argtypes = [C.c_void_p]
        lib.sst_set_connection.argtypes = [C.c_void_p, C.c_int32, C.c_int, C.c_double, C.c_double]
        lib.sst_seed_area.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double]
        lib.sst_step.argtypes = [C.c_void_p, C.c_int64]
        lib.sst_get_record.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.sst_readouts.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.sst_foundered.argtypes = [C.c_void_p]
        _tangent_lib = lib
    return _tangent_lib


class Tangent:
    """The tangent-linear restatement (oracle/sinksim_tangent.cpp): the portable step over dual numbers carrying
    derivatives with respect to up to 10 parameters that enter through connection areas."""

    def __init__(self, ship, sim):
        tl = tangent_lib()
        self.nodes = len(ship["mu"])
        self.nconn = len(sim["ca"])
        S, M = _structs(ship, sim)
        self.tl = tl
        self.t = tl.sst_create(C.byref(S), C.byref(M))

    def __del__(self):
        if getattr(self, "t", None):
            self.tl.sst_destroy(self.t)
            self.t = None

    def set_connection(self, c, enabled=-1, area=float("nan"), tOn=float("nan")):
        self.tl.sst_set_connection(self.t, c, enabled, area, tOn)

    def seed_area(self, c, p, g):
        self.tl.sst_seed_area(self.t, c, p, g)

    def step(self, n=1):
        self.tl.sst_step(self.t, n)

    def record(self, tangents=False):
        r = np.empty(10 + 5 * self.nodes)
        d = np.empty((TANGENT_PARAMS, r.size))
        self.tl.sst_get_record(self.t, _p(r, C.c_double), _p(d, C.c_double))
        return (r, d) if tangents else r

    def readouts(self, tangents=False):
        r = np.empty(7)
        d = np.empty((TANGENT_PARAMS, 7))
        self.tl.sst_readouts(self.t, _p(r, C.c_double), _p(d, C.c_double))
        return (r, d) if tangents else r

    def foundered(self):
        return bool(self.tl.sst_foundered(self.t))


# ----------------------------------------------------------------------------------------------- the adjoint on the host

_adjoint_host_lib = None


def adjoint_host_gradient(ship, sim, en, area, t_on, steps, sample_steps, trim_target, heave_target):
    """The product's reverse step run on the CPU (oracle/adjoint_host.cpp) over the C restatement's tapes: the
    trajectory objective sum_k (trim - trim_k)^2 + (heave - heave_k)^2 at the states after sample_steps[k] steps and its
    gradient with respect to every connection area. Returns (J, grad, error bits)."""
    global _adjoint_host_lib
    if _adjoint_host_lib is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libsinksim_adjoint_host.so"))
        lib.ssa_gradient.restype = C.c_int
        lib.ssa_gradient.argtypes = [C.POINTER(_Ship), C.POINTER(_Sim), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]
        _adjoint_host_lib = lib
    S, M = _structs(ship, sim)
    en = np.ascontiguousarray(en, dtype=np.uint8)
    area = f64(area)
    t_on = f64(t_on)
    ss = np.ascontiguousarray(sample_steps, dtype=np.int64)
    tt = f64(trim_target)
    ht = f64(heave_target)
    grad = np.zeros(len(sim["ca"]))
    J = C.c_double()
    err = _adjoint_host_lib.ssa_gradient(C.byref(S), C.byref(M), en.ctypes.data, area.ctypes.data, t_on.ctypes.data, int(steps), ss.size,
                                         ss.ctypes.data, tt.ctypes.data, ht.ctypes.data, C.byref(J), grad.ctypes.data)
    return J.value, grad, err


def tangent_gradient(ship, sim, en, area, t_on, conns, steps, sample_steps, trim_target, heave_target):
    """d J / d area[c] for the connections `conns` (at most 10) by the tangent-linear restatement, and J."""
    t = Tangent(ship, sim)
    for c in range(len(sim["ca"])):
        t.set_connection(c, enabled=int(en[c]), area=float(area[c]), tOn=float(t_on[c]))
    for p, c in enumerate(conns):
        t.seed_area(int(c), p, 1.0)
    order = np.argsort(sample_steps, kind="stable")
    done, J = 0, 0.0
    g = np.zeros(TANGENT_PARAMS)
    vals = {}
    for k in order:
        s = min(int(sample_steps[k]), steps)
        if s > done:
            t.step(s - done)
            done = s
        r, d = t.readouts(tangents=True)
        vals[k] = (r, d)
    for k in range(len(sample_steps)):
        r, d = vals[k]
        trim, heave = r[1], 0.5 * (r[5] + r[6])
        dtrim, dheave = d[:, 1], 0.5 * (d[:, 5] + d[:, 6])
        J += (trim - trim_target[k]) ** 2 + (heave - heave_target[k]) ** 2
        g += 2 * (trim - trim_target[k]) * dtrim + 2 * (heave - heave_target[k]) * dheave
    return J, g[:len(conns)]


# ----------------------------------------------------------------------------------------------- the reference engine

_ref_lib = None


def ref_lib():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(os.path.join(REF_DIR, "libsinksim_ref.so"))
        lib.ssref_last_error.restype = C.c_char_p
        lib.ssref_open.restype = C.c_void_p
        lib.ssref_open.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
        lib.ssref_close.argtypes = [C.c_void_p]
        lib.ssref_nodes.argtypes = [C.c_void_p]
        lib.ssref_connections.argtypes = [C.c_void_p]
        lib.ssref_set_connection.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]
        lib.ssref_apply_sweep_instance.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        lib.ssref_step.argtypes = [C.c_void_p, C.c_longlong]
        lib.ssref_state.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.ssref_restore.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.ssref_evaluate_hydro.argtypes = [C.c_void_p]
        lib.ssref_events.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        lib.ssref_foundered.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.ssref_readouts.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.ssref_run.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.c_int]
        lib.ssref_time_steps.restype = C.c_longlong
        lib.ssref_time_steps.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_longlong, C.c_int, C.POINTER(C.c_double)]
        _ref_lib = lib
    return _ref_lib


class RefSim:
    """The reference CPU engine (sinksim::Simulation) on one compiled ship and sim."""

    def __init__(self, ship_path, sim_path, numerics="portable"):
        self.lib = ref_lib()
        self.h = self.lib.ssref_open(ship_path.encode(), sim_path.encode(), numerics.encode())
        if not self.h:
            raise RuntimeError(self.lib.ssref_last_error().decode())
        self.nodes = self.lib.ssref_nodes(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ssref_close(self.h)
            self.h = None

    def _ok(self, rc):
        if rc < 0:
            raise RuntimeError(self.lib.ssref_last_error().decode())
        return rc

    def set_connection(self, c, enabled=-1, area=float("nan"), tOn=float("nan")):
        self._ok(self.lib.ssref_set_connection(self.h, c, enabled, area, tOn))

    def apply_sweep_instance(self, sweep_path, i):
        self._ok(self.lib.ssref_apply_sweep_instance(self.h, sweep_path.encode(), i))

    def step(self, n=1):
        self._ok(self.lib.ssref_step(self.h, n))

    def record(self):
        r = np.empty(10 + 5 * self.nodes)
        self.lib.ssref_state(self.h, _p(r, C.c_double))
        return r

    def restore(self, rec):
        rec = f64(rec)
        self._ok(self.lib.ssref_restore(self.h, _p(rec, C.c_double)))

    def readouts(self):
        r = np.empty(7)
        self.lib.ssref_readouts(self.h, _p(r, C.c_double))
        return r

    def events(self):
        buf = np.empty(3 * 1024)
        n = self._ok(self.lib.ssref_events(self.h, _p(buf, C.c_double), 1024))
        return [(buf[3 * i], int(buf[3 * i + 1]), int(buf[3 * i + 2])) for i in range(n)]

    def foundered(self):
        t = C.c_double()
        f = self.lib.ssref_foundered(self.h, C.byref(t))
        return bool(f), t.value

    def run(self, tMax, every, stop_when_stable=False, rule=None, cap=4096):
        """Simulation::run; returns (summary dict, curve array (records, 7))."""
        summary = np.zeros(5)
        curve = np.empty((cap, 7))
        rule_arr = f64(rule) if rule is not None else None
        rp = _p(rule_arr, C.c_double) if rule_arr is not None else None
        n = self._ok(self.lib.ssref_run(self.h, tMax, every, 1 if stop_when_stable else 0, rp, _p(summary, C.c_double),
                                        _p(curve, C.c_double), cap))
        return dict(steps=int(summary[0]), foundered=bool(summary[1]), founderT=summary[2], tEnd=summary[3],
                    retired=int(summary[4])), curve[:min(n, cap)].copy()


def ref_time_steps(ship_path, sim_path, numerics, count, max_steps, threads):
    """Times the reference CPU engine over a bounded sample; returns (steps, seconds)."""
    lib = ref_lib()
    sec = C.c_double()
    steps = lib.ssref_time_steps(ship_path.encode(), sim_path.encode(), numerics.encode(), count, max_steps, threads, C.byref(sec))
    if steps < 0:
        raise RuntimeError(lib.ssref_last_error().decode())
    return steps, sec.value


def ref_tool(name):
    return os.path.join(REF_DIR, name)


def fdlibm_ref():
    lib = C.CDLL(os.path.join(REF_DIR, "libfdlibm_ref.so"))
    for fn in ("fdlibm_sin", "fdlibm_cos"):
        getattr(lib, fn).restype = C.c_double
        getattr(lib, fn).argtypes = [C.c_double]
    lib.fdlibm_pow.restype = C.c_double
    lib.fdlibm_pow.argtypes = [C.c_double, C.c_double]
    lib.fdlibm_scalbn.restype = C.c_double
    lib.fdlibm_scalbn.argtypes = [C.c_double, C.c_int]
    return lib
