"""sinksim_b200: a B200-native batch engine for ship flooding simulation.

A drop-in for the batch path of the reference sinksim engine: it reads the same compiled ship, sim and sweep files,
computes the same "portable" / "portable32" numerics bit for bit, and writes the same batch-results and traces.
This module is the Python face of the C ABI in include/sinksim_b200.h (libsinksim_b200.so, built in the source tree
by ``python -m sinksim_b200.build``). It mirrors the reference's ``cuda::Batch`` (engine/include/sinksim/cuda/batch.hpp)
and the two batch tools (apps/sinksim_cuda_run.cpp, apps/sinksim_sweep.cpp).

There is no CPU fallback: without the built library or a CUDA device every entry point raises.
"""
import ctypes as C
import os

import numpy as np

__all__ = ["Batch", "Adjoint", "SinksimError", "available", "device_info", "run_sweep", "compare_results", "portable_math", "library_path",
           "STOP_REASONS", "NUMERICS"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsinksim_b200.so")
NUMERICS = {"portable": 0, "portable32": 1}
HEALTH_NON_FINITE = 1
HEALTH_STAGE_TIMEOUT = 2
STOP_REASONS = {0: "running", 1: "foundered", 2: "tmax", 3: "sink-rule", 4: "settle-rule", 5: "stable"}
_ERRORS = {-1: "invalid argument", -2: "runtime error", -3: "call out of order", -4: "unsupported", -5: "no CUDA device"}


class SinksimError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{_ERRORS.get(code, code)}: {message}")
        self.code = code


class _Options(C.Structure):
    _fields_ = [("count", C.c_int32), ("numerics", C.c_int32), ("traced_instances", C.c_int32), ("dense_steps", C.c_int32),
                ("sample_every", C.c_double), ("curve_every", C.c_double), ("t_max", C.c_double), ("steps_per_launch", C.c_int64),
                ("team_warps", C.c_int32), ("tail_team_warps", C.c_int32), ("teams_per_block", C.c_int32), ("yield_below", C.c_int32),
                ("blocks", C.c_int32), ("device", C.c_int32), ("rule_enabled", C.c_int32),
                ("rule_pitch", C.c_double), ("rule_x", C.c_double), ("rule_y", C.c_double), ("rule_z", C.c_double),
                ("rule_wth", C.c_double), ("rule_settle", C.c_double), ("stop_when_stable", C.c_int32), ("handover_factor", C.c_double),
                ("claim_by_index", C.c_int32), ("stage_columns", C.c_int32)]


class _DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("major", C.c_int32), ("minor", C.c_int32), ("multiprocessors", C.c_int32),
                ("global_memory", C.c_uint64), ("shared_per_block_optin", C.c_uint64), ("runtime_version", C.c_int32),
                ("driver_version", C.c_int32)]


class _Summary(C.Structure):
    _fields_ = [("foundered", C.c_int32), ("stop_reason", C.c_int32), ("founder_t", C.c_double), ("t_end", C.c_double),
                ("steps", C.c_int64), ("event_count", C.c_int32), ("curve_count", C.c_int32), ("outputs", C.c_double * 7)]


class _LaunchInfo(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("team_warps", "teams_per_block", "blocks", "blocks_per_sm", "yield_below", "tail_team_warps",
                                         "tail_teams_per_block", "tail_blocks", "tail_blocks_per_sm")] + [("slot_bytes", C.c_uint64), ("phases", C.c_int32),
                                                                                            ("kernels", C.c_int32), ("staged_phases", C.c_int32)]


_lib = None

_SIGNATURES = {
    "ssb_last_error": (C.c_char_p, []),
    "ssb_version": (C.c_char_p, []),
    "ssb_available": (C.c_int, [C.c_char_p, C.c_size_t]),
    "ssb_get_device_info": (C.c_int, [C.c_int32, C.POINTER(_DeviceInfo)]),
    "ssb_batch_options_init": (None, [C.POINTER(_Options)]),
    "ssb_batch_create": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_Options), C.POINTER(C.c_void_p)]),
    "ssb_batch_destroy": (None, [C.c_void_p]),
    "ssb_batch_nodes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ssb_batch_launch_info": (C.c_int, [C.c_void_p, C.POINTER(_LaunchInfo)]),
    "ssb_batch_restore": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "ssb_batch_set_connection_enabled": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "ssb_batch_set_connection_area": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double]),
    "ssb_batch_set_connection_activation": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_double]),
    "ssb_batch_set_connection_areas": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "ssb_batch_set_claim_order": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "ssb_batch_apply_sweep": (C.c_int, [C.c_void_p, C.c_char_p]),
    "ssb_fleet_create": (C.c_int, [C.c_int32, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), C.POINTER(C.c_int32), C.c_void_p, C.POINTER(C.c_void_p)]),
    "ssb_batch_instance_shape": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ssb_batch_apply_sweep_range": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int32]),
    "ssb_batch_run": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "ssb_batch_upload": (C.c_int, [C.c_void_p]),
    "ssb_batch_reset": (C.c_int, [C.c_void_p]),
    "ssb_batch_launch": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "ssb_batch_download": (C.c_int, [C.c_void_p]),
    "ssb_batch_transfer_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ssb_batch_total_steps": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "ssb_batch_phase_stats": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_int64)]),
    "ssb_batch_summary": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(_Summary)]),
    "ssb_batch_state": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "ssb_batch_events": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32,
                                   C.POINTER(C.c_int32)]),
    "ssb_batch_curve": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_int32)]),
    "ssb_batch_final_readouts": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double)]),
    "ssb_batch_save_trace": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p]),
    "ssb_batch_save_results": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p]),
    "ssb_run_sweep": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "ssb_run_sweep_range": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.c_int32, C.c_char_p,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "ssb_compare_results": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]),
    "ssb_portable_math_host": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64]),
    "ssb_portable_math_device": (C.c_int, [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int64]),
    "ssb_measure_add_mul_peak": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_double)]),
    "ssb_batch_run_noalloc": (C.c_int, [C.c_void_p, C.c_int32] + [C.c_void_p] * 13),
    "ssb_fnv1a64": (C.c_uint64, [C.c_uint64, C.c_void_p, C.c_size_t]),
    "ssb_adjoint_create": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "ssb_adjoint_destroy": (None, [C.c_void_p]),
    "ssb_adjoint_set_connection_enabled": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32]),
    "ssb_adjoint_set_connection_areas": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "ssb_adjoint_set_objective": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ssb_adjoint_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]),
    "ssb_adjoint_samples": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "ssb_adjoint_phase_times": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ssb_adjoint_set_tape_budget": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ssb_adjoint_set_claim_order": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "ssb_adjoint_recomputed_steps": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ssb_adjoint_ring_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "ssb_adjoint_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64)]),
    "ssb_check_model": (C.c_int, [C.c_char_p, C.c_char_p]),
    "ssb_batch_health": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "ssb_check_sweep": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p]),
    "ssb_launch_plan": (C.c_int, [C.POINTER(_Options), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]),
}

PLAN_KINDS = {0: "start_run", 1: "claim_order", 2: "phase"}


def launch_plan(yield_below, steps_per_launch=0, claim_by_index=False):
    """The kernels one run to the end captures in its CUDA graph, for launch phases whose hand-over bounds are
    `yield_below` (one per phase, the last 0): [(kind, phase), ...] with kind start_run (1 kernel), claim_order (the 2
    kernels that rank the unfinished instances) or phase (the phase's batch kernel). Host-only."""
    o = _Options()
    lib().ssb_batch_options_init(C.byref(o))
    o.steps_per_launch = steps_per_launch
    o.claim_by_index = 1 if claim_by_index else 0
    y = np.ascontiguousarray(yield_below, dtype=np.int32)
    cap = 2 * y.size + 1
    kinds = np.empty(cap, dtype=np.int32)
    phases = np.empty(cap, dtype=np.int32)
    n = C.c_int32()
    _check(lib().ssb_launch_plan(C.byref(o), y.size, y.ctypes.data, kinds.ctypes.data, phases.ctypes.data, cap, C.byref(n)))
    return [(PLAN_KINDS[int(kinds[i])], int(phases[i])) for i in range(n.value)]


def fnv1a64(state, data):
    """FNV-1a 64-bit of the bytes `data`, continuing from `state` (the compiled files' hash)."""
    buf = bytes(data)
    return int(lib().ssb_fnv1a64(state, buf, len(buf)))


def add_mul_peak(fp64=True, device=0):
    """Measured separately-rounded add+multiply rate of the device (operations per second)."""
    v = C.c_double()
    _check(lib().ssb_measure_add_mul_peak(1 if fp64 else 0, device, C.byref(v)))
    return v.value


def check_model(ship_path, sim_path, sweep_path=None):
    """Verifies a compiled ship and sim (and a sweep file against them) without running anything: formats, lengths,
    ranges, every hash and the pairing. Raises SinksimError with the first problem."""
    if sweep_path is None:
        _check(lib().ssb_check_model(_b(ship_path), _b(sim_path)))
    else:
        _check(lib().ssb_check_sweep(_b(ship_path), _b(sim_path), _b(sweep_path)))


def library_path():
    return LIB_PATH


def lib():
    """The loaded libsinksim_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sinksim_b200.build` (there is no CPU fallback)")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def _check(rc):
    if rc < 0:
        raise SinksimError(rc, lib().ssb_last_error().decode())
    return rc


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _b(s):
    return None if s is None else os.fsencode(s)


def available():
    """(ok, reason): is a CUDA device usable?"""
    why = C.create_string_buffer(512)
    ok = lib().ssb_available(why, 512)
    return bool(ok), why.value.decode()


def device_info(device=0):
    d = _DeviceInfo()
    _check(lib().ssb_get_device_info(device, C.byref(d)))
    return dict(name=d.name.decode(), major=d.major, minor=d.minor, multiprocessors=d.multiprocessors,
                global_memory=d.global_memory, shared_per_block_optin=d.shared_per_block_optin,
                runtime_version=d.runtime_version, driver_version=d.driver_version)


class Batch:
    """Many instances of one compiled ship and sim on one GPU (the reference's cuda::Batch).

    numerics: "portable" (double precision) or "portable32" (single-precision column partials).
    rule: optional dict(pitch=, x=, y=, z=, wth=, settle=) for the extra sink/settle retire rule.
    stage_columns: every block copies the column table into its shared memory and the buoyancy reads it from there
    (ssb_batch_options.stage_columns); the results are the same.
    """

    def __init__(self, ship_path, sim_path, count=1, numerics="portable32", traced_instances=0, dense_steps=400, sample_every=60.0,
                 curve_every=0.0, t_max=5 * 3600.0, steps_per_launch=0, team_warps=0, tail_team_warps=-1, teams_per_block=0, yield_below=-1,
                 blocks=0, device=0, rule=None, stop_when_stable=False, handover_factor=0.0, claim_by_index=False, stage_columns=False,
                 _fleet=None):
        if numerics not in NUMERICS:
            raise SinksimError(-4, f"numerics {numerics!r} is not available on the GPU (portable or portable32)")
        o = _Options()
        lib().ssb_batch_options_init(C.byref(o))
        o.count, o.numerics, o.traced_instances, o.dense_steps = count, NUMERICS[numerics], traced_instances, dense_steps
        o.sample_every, o.curve_every, o.t_max, o.steps_per_launch = sample_every, curve_every, t_max, steps_per_launch
        o.team_warps, o.tail_team_warps, o.teams_per_block, o.yield_below = team_warps, tail_team_warps, teams_per_block, yield_below
        o.blocks, o.device = blocks, device
        o.stop_when_stable = 1 if stop_when_stable else 0
        o.handover_factor = handover_factor
        o.claim_by_index = 1 if claim_by_index else 0
        o.stage_columns = 1 if stage_columns else 0
        if rule:
            o.rule_enabled = 1
            o.rule_pitch, o.rule_x, o.rule_y, o.rule_z = rule["pitch"], rule["x"], rule["y"], rule["z"]
            o.rule_wth, o.rule_settle = rule["wth"], rule["settle"]
        h = C.c_void_p()
        if _fleet is None:
            _check(lib().ssb_batch_create(_b(ship_path), _b(sim_path), C.byref(o), C.byref(h)))
        else:
            models, instance_model = _fleet
            ships = (C.c_char_p * len(models))(*[_b(s) for s, _ in models])
            sims = (C.c_char_p * len(models))(*[_b(m) for _, m in models])
            im = (C.c_int32 * count)(*[int(v) for v in instance_model])
            _check(lib().ssb_fleet_create(len(models), ships, sims, im, C.byref(o), C.byref(h)))
        self._h = h
        self.count = count
        self.numerics = numerics
        n, c = C.c_int32(), C.c_int32()
        _check(lib().ssb_batch_nodes(self._h, C.byref(n), C.byref(c)))
        self.nodes, self.connections = n.value, c.value

    @classmethod
    def fleet(cls, models, instance_model, **options):
        """Instances of several models in one batch: models = [(ship_path, sim_path), ...], instance_model[i] = the model
        of instance i. Options as for Batch (count is len(instance_model)); no traces, sweeps or batch-results files."""
        instance_model = list(instance_model)
        options.pop("count", None)
        return cls(None, None, count=len(instance_model), _fleet=(list(models), instance_model), **options)

    def instance_shape(self, instance):
        """(model index, nodes, connections) of one instance."""
        m, n, c = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().ssb_batch_instance_shape(self._h, instance, C.byref(m), C.byref(n), C.byref(c)))
        return m.value, n.value, c.value

    def close(self):
        if getattr(self, "_h", None):
            lib().ssb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def launch_info(self):
        li = _LaunchInfo()
        _check(lib().ssb_batch_launch_info(self._h, C.byref(li)))
        return {k: getattr(li, k) for k, _ in _LaunchInfo._fields_}

    # per-instance setup
    def restore(self, instance, record):
        rec = np.ascontiguousarray(record, dtype=np.float64)
        if rec.size != 10 + 5 * self.nodes:
            raise SinksimError(-1, f"a state record has {10 + 5 * self.nodes} values, got {rec.size}")
        _check(lib().ssb_batch_restore(self._h, instance, _dptr(rec)))

    def set_connection_enabled(self, instance, connection, enabled):
        _check(lib().ssb_batch_set_connection_enabled(self._h, instance, connection, 1 if enabled else 0))

    def set_connection_area(self, instance, connection, area):
        _check(lib().ssb_batch_set_connection_area(self._h, instance, connection, float(area)))

    def set_connection_activation(self, instance, connection, t_on):
        _check(lib().ssb_batch_set_connection_activation(self._h, instance, connection, float(t_on)))

    def set_connection_areas(self, first, connections, areas):
        """Areas of a block of instances in one call: areas[i, j] (a [count, len(connections)] array) becomes the area
        of connection connections[j] of instance first + i."""
        conns = np.ascontiguousarray(connections, dtype=np.int32)
        a = np.ascontiguousarray(areas, dtype=np.float64)
        if a.ndim != 2 or a.shape[1] != conns.size:
            raise SinksimError(-1, f"areas must be [count, {conns.size}], got {list(a.shape)}")
        _check(lib().ssb_batch_set_connection_areas(self._h, int(first), a.shape[0], conns.size,
                                                     conns.ctypes.data, a.ctypes.data))

    def set_claim_order(self, order):
        """The first launch phase claims the instances in this order (a permutation of range(count)), e.g. the
        longest expected runs first."""
        o = np.ascontiguousarray(order, dtype=np.int32)
        _check(lib().ssb_batch_set_claim_order(self._h, o.ctypes.data, o.size))

    def apply_sweep(self, sweep_path, first=None):
        """Instance i takes sweep instance i; with `first`, sweep instance first + i (a shard of a longer sweep)."""
        if first is None:
            _check(lib().ssb_batch_apply_sweep(self._h, _b(sweep_path)))
        else:
            _check(lib().ssb_batch_apply_sweep_range(self._h, _b(sweep_path), int(first)))

    # running
    def run(self):
        s = C.c_double()
        _check(lib().ssb_batch_run(self._h, C.byref(s)))
        return s.value

    def reset(self):
        """Make the batch runnable again from its staged inputs."""
        _check(lib().ssb_batch_reset(self._h))

    def upload(self):
        _check(lib().ssb_batch_upload(self._h))

    def launch(self):
        ms = C.c_float()
        _check(lib().ssb_batch_launch(self._h, C.byref(ms)))
        return ms.value

    def download(self):
        _check(lib().ssb_batch_download(self._h))

    def health(self):
        """Flags of the last run: 0, or 1 when an instance's state went NaN or infinite (HEALTH_NON_FINITE), 2 when a
        block read the column table from global memory because its staged copy did not arrive in time
        (HEALTH_STAGE_TIMEOUT)."""
        f = C.c_int32()
        _check(lib().ssb_batch_health(self._h, C.byref(f)))
        return f.value

    def transfer_bytes(self):
        a, b = C.c_uint64(), C.c_uint64()
        _check(lib().ssb_batch_transfer_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    # results
    def total_steps(self):
        s = C.c_int64()
        _check(lib().ssb_batch_total_steps(self._h, C.byref(s)))
        return s.value

    def phase_stats(self):
        """The last launch by phase: [{team_warps, device_ms, steps}, ...] (CUDA-event time of each phase's kernel)."""
        out = []
        for k in range(self.launch_info()["phases"]):
            w, ms, st = C.c_int32(), C.c_float(), C.c_int64()
            _check(lib().ssb_batch_phase_stats(self._h, k, C.byref(w), C.byref(ms), C.byref(st)))
            out.append({"team_warps": w.value, "device_ms": ms.value, "steps": st.value})
        return out

    def summary(self, instance):
        s = _Summary()
        _check(lib().ssb_batch_summary(self._h, instance, C.byref(s)))
        return dict(foundered=bool(s.foundered), stop=STOP_REASONS.get(s.stop_reason, s.stop_reason), founder_t=s.founder_t,
                    t_end=s.t_end, steps=s.steps, event_count=s.event_count, curve_count=s.curve_count, outputs=list(s.outputs))

    def state(self, instance):
        r = np.empty(10 + 5 * self.instance_shape(instance)[1])
        _check(lib().ssb_batch_state(self._h, instance, _dptr(r)))
        return r

    def events(self, instance, cap=4096):
        t = np.empty(cap)
        ids = np.empty(cap, dtype=np.int32)
        kinds = np.empty(cap, dtype=np.int32)
        n = C.c_int32()
        _check(lib().ssb_batch_events(self._h, instance, _dptr(t), ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                      kinds.ctypes.data_as(C.POINTER(C.c_int32)), cap, C.byref(n)))
        k = min(n.value, cap)
        return [(float(t[i]), int(ids[i]), int(kinds[i])) for i in range(k)]

    def curve(self, instance, cap=None):
        cap = cap or self.summary(instance)["curve_count"]
        out = np.empty((max(cap, 1), 7))
        n = C.c_int32()
        _check(lib().ssb_batch_curve(self._h, instance, _dptr(out), cap, C.byref(n)))
        return out[:min(n.value, cap)].copy()

    def final_readouts(self, instance):
        r = np.empty(7)
        _check(lib().ssb_batch_final_readouts(self._h, instance, _dptr(r)))
        return r

    def save_trace(self, instance, path):
        _check(lib().ssb_batch_save_trace(self._h, instance, _b(path)))

    def save_results(self, path, sweep_path=None):
        _check(lib().ssb_batch_save_results(self._h, _b(sweep_path), _b(path)))

    def run_noalloc(self, count, en, area, t_on, state, vol, level, cx, cy, cz, final_readouts, steps, stop_reason, stream=None):
        """Runs `count` instances of this batch's model in the caller's device memory without allocating any (see
        ssb_batch_run_noalloc in include/sinksim_b200.h). Every buffer argument is a device address (int); returns
        once the work is queued on `stream` (a cudaStream_t as int, or None for the default stream)."""
        _check(lib().ssb_batch_run_noalloc(self._h, count, en, area, t_on, state, vol, level, cx, cy, cz, final_readouts, steps, stop_reason,
                                           stream))


class Adjoint:
    """Objective and gradient of a trajectory misfit for many instances of one compiled model, by the engine's discrete
    adjoint (FP64, checkpoints every `checkpoint_every` steps, see include/sinksim_b200.h, ssb_adjoint_*).

    Instance i runs from the compiled initial state until t_max or its founder; its objective is
    sum_k (trim_k - trim_target[i, k])^2 + (heave_k - heave_target[i, k])^2 at the sample times, and run() returns it
    with its gradient with respect to every connection area."""

    def __init__(self, ship_path, sim_path, count=1, t_max=7920.0, checkpoint_every=256, team_warps=0, device=0, tape_budget=0):
        h = C.c_void_p()
        _check(lib().ssb_adjoint_create(_b(ship_path), _b(sim_path), count, float(t_max), checkpoint_every, team_warps, device, C.byref(h)))
        self._h = h
        self.count = count
        nc = C.c_int32()
        _check(lib().ssb_adjoint_info(self._h, C.byref(nc), None, None, None, None))
        self.connections = nc.value
        self.nsamples = 0
        if tape_budget:
            self.set_tape_budget(tape_budget)

    def set_claim_order(self, order):
        """The order in which the teams claim the instances (a permutation of range(count)), or None for index order;
        see ssb_adjoint_set_claim_order. The results do not depend on it."""
        if order is None:
            _check(lib().ssb_adjoint_set_claim_order(self._h, None, 0))
            return
        o = np.ascontiguousarray(order, dtype=np.int32)
        _check(lib().ssb_adjoint_set_claim_order(self._h, o.ctypes.data, o.size))

    def set_tape_budget(self, nbytes):
        """Device memory for step records, all teams together (0: a whole run's, within half the free memory at the
        next run); see ssb_adjoint_set_tape_budget. The results do not depend on it."""
        _check(lib().ssb_adjoint_set_tape_budget(self._h, int(nbytes)))

    def recomputed_steps(self):
        """Steps each instance recomputed from its checkpoints in the last run [count]."""
        n = np.empty(self.count, dtype=np.int64)
        _check(lib().ssb_adjoint_recomputed_steps(self._h, n.ctypes.data))
        return n

    def ring_bytes(self):
        """Each team's ring of step records in the last run, bytes."""
        b = C.c_uint64()
        _check(lib().ssb_adjoint_ring_bytes(self._h, C.byref(b)))
        return b.value

    def close(self):
        if getattr(self, "_h", None):
            lib().ssb_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_connection_enabled(self, instance, connection, enabled):
        _check(lib().ssb_adjoint_set_connection_enabled(self._h, instance, connection, 1 if enabled else 0))

    def set_connection_areas(self, first, connections, areas):
        conns = np.ascontiguousarray(connections, dtype=np.int32)
        a = np.ascontiguousarray(areas, dtype=np.float64)
        if a.ndim != 2 or a.shape[1] != conns.size:
            raise SinksimError(-1, f"areas must be [count, {conns.size}], got {list(a.shape)}")
        _check(lib().ssb_adjoint_set_connection_areas(self._h, int(first), a.shape[0], conns.size, conns.ctypes.data, a.ctypes.data))

    def set_objective(self, times, trim_target, heave_target):
        t = np.ascontiguousarray(times, dtype=np.float64)
        tr = np.ascontiguousarray(np.broadcast_to(np.asarray(trim_target, dtype=np.float64), (self.count, t.size)))
        hv = np.ascontiguousarray(np.broadcast_to(np.asarray(heave_target, dtype=np.float64), (self.count, t.size)))
        _check(lib().ssb_adjoint_set_objective(self._h, t.size, t.ctypes.data, tr.ctypes.data, hv.ctypes.data))
        self.nsamples = t.size

    def run(self):
        """(J [count], grad [count, connections], steps [count], error [count], device ms)."""
        J = np.empty(self.count)
        g = np.empty((self.count, self.connections))
        steps = np.empty(self.count, dtype=np.int64)
        err = np.empty(self.count, dtype=np.int32)
        ms = C.c_float()
        _check(lib().ssb_adjoint_run(self._h, J.ctypes.data, g.ctypes.data, steps.ctypes.data, err.ctypes.data, C.byref(ms)))
        return J, g, steps, err, ms.value

    def samples(self):
        """The last run's (trim, heave) at the sample times, [count, n] each."""
        tr = np.empty((self.count, self.nsamples))
        hv = np.empty((self.count, self.nsamples))
        _check(lib().ssb_adjoint_samples(self._h, tr.ctypes.data, hv.ctypes.data))
        return tr, hv

    def phase_times(self):
        """The last run's time per instance [count, 3] in seconds of its team: forward, recomputation, reverse."""
        ns = np.empty((self.count, 3), dtype=np.int64)
        _check(lib().ssb_adjoint_phase_times(self._h, ns.ctypes.data))
        return ns * 1e-9

    def info(self):
        nc, w, t = C.c_int32(), C.c_int32(), C.c_int32()
        up, down = C.c_uint64(), C.c_uint64()
        _check(lib().ssb_adjoint_info(self._h, C.byref(nc), C.byref(w), C.byref(t), C.byref(up), C.byref(down)))
        return dict(connections=nc.value, team_warps=w.value, teams=t.value, h2d_bytes=up.value, d2h_bytes=down.value)


def run_sweep(ship_path, sim_path, sweep_path, numerics="portable32", results_path=None):
    """sinksim_cuda_run --sweep in one call; returns (aggregate steps, wall seconds)."""
    steps, secs = C.c_int64(), C.c_double()
    _check(lib().ssb_run_sweep(_b(ship_path), _b(sim_path), _b(sweep_path), numerics.encode(), _b(results_path), C.byref(steps), C.byref(secs)))
    return steps.value, secs.value


def run_sweep_range(ship_path, sim_path, sweep_path, first, count=-1, numerics="portable32", results_path=None, device=0):
    """run_sweep on sweep instances [first, first + count) on one device (a shard); returns (steps, wall seconds)."""
    steps, secs = C.c_int64(), C.c_double()
    _check(lib().ssb_run_sweep_range(_b(ship_path), _b(sim_path), _b(sweep_path), numerics.encode(), int(first), int(count), int(device),
                                     _b(results_path), C.byref(steps), C.byref(secs)))
    return steps.value, secs.value


def compare_results(a_path, b_path):
    """Exact value-for-value comparison of two batch-results files; returns (compared, differing, first difference)."""
    comp, diff = C.c_uint64(), C.c_uint64()
    first = C.create_string_buffer(1024)
    _check(lib().ssb_compare_results(_b(a_path), _b(b_path), C.byref(comp), C.byref(diff), first, 1024))
    return comp.value, diff.value, first.value.decode()


_OPS = {"sin": 0, "cos": 1, "pow": 2, "scalbn": 3}


def portable_math(op, x, y=None, device=True):
    """The engine's portable sin/cos/pow/scalbn on arrays, evaluated on the GPU (device=True) or the host."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    yy = None if y is None else np.ascontiguousarray(np.broadcast_to(np.asarray(y, dtype=np.float64), x.shape))
    out = np.empty_like(x)
    f = lib().ssb_portable_math_device if device else lib().ssb_portable_math_host
    _check(f(_OPS[op], _dptr(x), None if yy is None else _dptr(yy), _dptr(out), x.size))
    return out
