"""Synthetic hull compiler: writes a parametric liner as a compiled ship and sim in the reference's formats.

The reference builds its ships in its JS oracle and exports them (tools/js/export_compiled.js; the node, connection
and mass recipe in oracle/js/core/core.js:192-330, 716-824). This module builds a hull from a few dimensions instead:

* a grid of NX x NY vertical columns over L x B; half-breadth constant over the middle 60% of the length with a
  parabolic taper to zero at both ends (each column's footprint is its cell's width inside the hull); bottoms rise
  quadratically over the end 20% on each side; depth D at midships rising linearly to D + sheer at the ends; keel z = 0;
* n_comp watertight compartments along the length x n_decks decks: one space (node) per compartment and deck, each
  its own free-surface group; segments are the parts of the compartment's columns between the deck heights;
* per space: permeability mu, capacity mu x sum(dxdy x height), minimum flow area max(4, 0.15 mu x footprint) and
  pressed-up area max(1, 0.03 x footprint);
* connections: bulkhead-top weirs and doors (area U(1, 3) m2, sill U(0, 1) m, closed) between longitudinally adjacent
  spaces (the bulkhead weirs' crest is the bulkhead deck's height where the deck is lower), two deck openings
  (U(0.5, 4) m2) between each space and the one above plus extra hatches amidships, weather-deck openings to the sea,
  and breaches below the waterline in the forward compartments, on alternating sides (the last ones closed);
* mass for an even-keel draft T with metacentric height GM; inertia, added mass and damping from critical-damping
  fractions of the intact hydrostatics (the reference's recipe, core.js:800-816); the state at rest at that draft;
* every hashed array carries the FNV-1a 64-bit hash the loader verifies (hashing order of export_compiled.js:24-33,
  85-103; -0 written as 0).

    python -m sinksim_b200.hullgen --out DIR [--seed 20261203] [--id liner269]

writes DIR/<id>.ship.json and DIR/<id>.sim.json. The defaults are the 269 x 28 m, 4,408-column, 64-space,
290-connection liner.
"""
import argparse
import json
import math
import os
import sys

import numpy as np

RHO, GRAV = 1025.0, 9.81
KIND_NAMES = ["door", "over", "down", "xlow", "xmerge", "xup", "top", "breach", "open"]
K_DOOR, K_OVER, K_DOWN, K_TOP, K_BREACH, K_OPEN = 0, 1, 2, 6, 7, 8
ORIFICE, WEIR = 0, 1
TOP_OPEN_SHARE = 0.05  # weir width of a compartment's weather-deck openings together: this share of its length
FNV_OFFSET, FNV_PRIME, MASK64 = 0xCBF29CE484222325, 0x100000001B3, (1 << 64) - 1


# ------------------------------------------------------------------------------------------ hashing

def _packed(kind, values):
    if kind == "f64":
        a = np.asarray(values, dtype="<f8").copy()
        a[a == 0] = 0.0  # JSON cannot hold -0
        return a.tobytes()
    if kind == "i32":
        return np.asarray(values, dtype="<i4").tobytes()
    if kind == "u8":
        return np.asarray(values, dtype=np.uint8).tobytes()
    raise ValueError(kind)


def _fnv(h, data):
    """FNV-1a 64-bit over data from state h: the library's routine when it is built, else the same loop here."""
    try:
        from . import fnv1a64
        return fnv1a64(h, data)
    except (ImportError, OSError, RuntimeError):
        for byte in data:
            h = ((h ^ byte) * FNV_PRIME) & MASK64
        return h


def hash_arrays(entries):
    """{name: hex} per array and "all" chained over them in order; entries = [(name, kind, values)]."""
    out = {}
    chain = FNV_OFFSET
    for name, kind, values in entries:
        data = _packed(kind, values)
        out[name] = f"{_fnv(FNV_OFFSET, data):016x}"
        chain = _fnv(chain, data)
    out["all"] = f"{chain:016x}"
    return out


# ------------------------------------------------------------------------------------------ the hull

class HullSpec:
    """Dimensions of a parametric liner (metres); the defaults are the 269 x 28 m benchmark liner."""

    def __init__(self, L=269.0, B=28.0, depth=18.0, sheer=4.0, nx=152, ny=29, n_comp=16, n_decks=4, draft=10.5, gm=0.8,
                 end_rise=3.0, breaches=6, reserve_breaches=2, breach_area=1.2, top_openings=4, extra_hatches=2, dt=0.25, bulkhead_top=13.5):
        self.L, self.B, self.depth, self.sheer = float(L), float(B), float(depth), float(sheer)
        self.nx, self.ny, self.n_comp, self.n_decks = int(nx), int(ny), int(n_comp), int(n_decks)
        self.draft, self.gm, self.end_rise = float(draft), float(gm), float(end_rise)
        self.breaches, self.reserve_breaches, self.breach_area, self.dt = int(breaches), int(reserve_breaches), float(breach_area), float(dt)
        self.top_openings, self.extra_hatches, self.bulkhead_top = int(top_openings), int(extra_hatches), float(bulkhead_top)

    def half_breadth(self, x):
        u = np.abs(x) / (0.5 * self.L)
        t = np.clip((u - 0.6) / 0.4, 0.0, 1.0)
        return 0.5 * self.B * (1.0 - t * t)

    def bottom(self, x):
        u = np.abs(x) / (0.5 * self.L)
        t = np.clip((u - 0.6) / 0.4, 0.0, 1.0)
        return self.end_rise * t * t

    def deck(self, x):
        return self.depth + self.sheer * np.abs(x) / (0.5 * self.L)

    def deck_floors(self):
        """Floor heights of the decks; the top deck reaches the weather deck."""
        h = self.depth * 0.75
        return [h * k / self.n_decks for k in range(self.n_decks)]


def build_columns(spec):
    dx, dy = spec.L / spec.nx, spec.B / spec.ny
    xs = 0.5 * spec.L - (np.arange(spec.nx) + 0.5) * dx          # bow first
    ys = -0.5 * spec.B + (np.arange(spec.ny) + 0.5) * dy
    cols = {k: [] for k in ("x", "y", "dxdy", "dx", "zlo", "zhi", "zone", "side")}
    comp_len = spec.L / spec.n_comp
    for x in xs:
        hb = float(spec.half_breadth(x))
        zone = min(int((0.5 * spec.L - x) // comp_len), spec.n_comp - 1)
        for y in ys:
            lo, hi = max(y - 0.5 * dy, -hb), min(y + 0.5 * dy, hb)
            w = hi - lo
            yc = 0.5 * (lo + hi)
            if w < 0.02:  # a cell beyond the hull: a thin column at the hull's edge keeps the grid whole
                w = 0.02
                yc = math.copysign(max(hb - 0.01, 0.0), y)
            cols["x"].append(float(x))
            cols["y"].append(float(yc))
            cols["dxdy"].append(float(dx * w))
            cols["dx"].append(float(dx))
            cols["zlo"].append(float(spec.bottom(x)))
            cols["zhi"].append(float(spec.deck(x)))
            cols["zone"].append(zone)
            cols["side"].append(0 if yc >= 0 else 1)
    cols["n"] = len(cols["x"])
    cols["dy"] = dy
    return cols


def build_nodes(spec, cols):
    floors = spec.deck_floors()
    nd = spec.n_decks
    lists = [[] for _ in range(spec.n_comp * nd)]
    for i in range(cols["n"]):
        k = cols["zone"][i]
        for d in range(nd):
            lo = max(cols["zlo"][i], floors[d])
            hi = cols["zhi"][i] if d == nd - 1 else min(cols["zhi"][i], floors[d + 1])
            if hi > lo + 1e-3:
                lists[k * nd + d].append((i, lo, hi))
    empty = [n for n, lst in enumerate(lists) if not lst]
    if empty:
        raise ValueError(f"spaces {empty} hold no part of any column: lower the bottom's end rise or the deck heights")
    seg_col, seg_a, seg_e, start, count = [], [], [], [], []
    for lst in lists:
        start.append(len(seg_col))
        count.append(len(lst))
        for i, a, e in lst:
            seg_col.append(i)
            seg_a.append(a)
            seg_e.append(e)
    mu, vmax, amin, aov, label = [], [], [], [], []
    for n, lst in enumerate(lists):
        k, d = divmod(n, nd)
        m = 0.85 if d == 0 else 0.95
        vm = sum(cols["dxdy"][i] * (e - a) for i, a, e in lst)
        fp = sum(cols["dxdy"][i] for i, _, _ in lst)
        mu.append(m)
        vmax.append(m * vm)
        amin.append(max(4.0, 0.15 * m * fp))
        aov.append(max(1.0, 0.03 * fp))
        label.append(f"C{k:02d}/deck{d}")
    return {"n": len(lists), "label": label, "mu": mu, "vmax": vmax, "amin": amin, "aov": aov, "segStart": start,
            "segCount": count}, {"n": len(seg_col), "col": seg_col, "a": seg_a, "e": seg_e}


def hydrostatics(cols, T):
    """Even-keel hydrostatics at draft T from the column table (the hull's buoyancy pass at zero attitude)."""
    x, y = np.array(cols["x"]), np.array(cols["y"])
    A, lo, hi = np.array(cols["dxdy"]), np.array(cols["zlo"]), np.array(cols["zhi"])
    dx = np.array(cols["dx"])
    s = np.clip(T - lo, 0.0, hi - lo)
    V = float(np.sum(A * s))
    lcb = float(np.sum(A * s * x)) / V
    kb = float(np.sum(A * s * (lo + 0.5 * s))) / V
    wp = (lo < T) & (hi > T)
    awp = float(np.sum(A[wp]))
    width = A / dx
    lcf = float(np.sum(A[wp] * x[wp])) / awp
    it = float(np.sum(A[wp] * (y[wp] ** 2 + width[wp] ** 2 / 12)))
    il = float(np.sum(A[wp] * ((x[wp] - lcf) ** 2 + dx[wp] ** 2 / 12)))
    return {"V": V, "LCB": lcb, "KB": kb, "Awp": awp, "LCF": lcf, "BM": it / V, "BML": il / V}


def ship_document(spec, ship_id, cols, nodes, segs, hyd):
    hashed = [
        ("columns.x", "f64", cols["x"]), ("columns.y", "f64", cols["y"]), ("columns.dxdy", "f64", cols["dxdy"]),
        ("columns.zlo", "f64", cols["zlo"]), ("columns.zhi", "f64", cols["zhi"]), ("columns.zone", "i32", cols["zone"]),
        ("columns.side", "i32", cols["side"]),
        ("nodes.mu", "f64", nodes["mu"]), ("nodes.vmax", "f64", nodes["vmax"]), ("nodes.amin", "f64", nodes["amin"]),
        ("nodes.aov", "f64", nodes["aov"]), ("nodes.segStart", "i32", nodes["segStart"]), ("nodes.segCount", "i32", nodes["segCount"]),
        ("segments.col", "i32", segs["col"]), ("segments.a", "f64", segs["a"]), ("segments.e", "f64", segs["e"]),
    ]
    return {
        "format": "sinksim.compiled-ship", "formatVersion": 1, "id": ship_id,
        "meta": {"title": f"parametric liner {spec.L:g} x {spec.B:g} m, {cols['n']} columns, {spec.n_comp} compartments x "
                          f"{spec.n_decks} decks", "generator": "sinksim_b200.hullgen", "spec": vars(spec)},
        "units": {"length": "m", "area": "m2", "volume": "m3", "mass": "kg", "time": "s", "angle": "rad"},
        "frame": {"x": "forward from amidships", "y": "to port", "z": "up from the keel baseline", "world": "sea surface at Z = 0",
                  "pitch": "bow down positive", "roll": "starboard down positive", "rotation": "R = Ry(pitch) * Rx(roll)",
                  "nodeIndex": "n = compartment * decks + deck; compartment 0 at the bow; deck 0 lowest"},
        "columns": cols, "nodes": nodes, "segments": segs,
        "hydrostatics": hyd,
        "hash": hash_arrays(hashed),
    }


# ------------------------------------------------------------------------------------------ the simulation

def build_connections(spec, cols, nodes, rng):
    nd, ncmp = spec.n_decks, spec.n_comp
    floors = spec.deck_floors()
    comp_len = spec.L / ncmp
    C = {k: [] for k in ("a", "b", "type", "x", "y", "z", "area", "coef", "kind", "idx", "en", "tOn", "skipGroup", "monitor")}

    def add(a, b, law, x, y, z, area, kind, idx, en, monitor=-1):
        for k, v in zip(("a", "b", "type", "x", "y", "z", "area", "coef", "kind", "idx", "en", "tOn", "skipGroup", "monitor"),
                        (a, b, law, x, y, z, area, 0.6, kind, idx, 1 if en else 0, 0.0, -1, monitor)):
            C[k].append(v)

    def deck_top(x, d):
        return float(spec.deck(x)) if d == nd - 1 else floors[d + 1]

    for bh in range(ncmp - 1):                       # bulkhead bh between compartments bh (forward) and bh + 1
        x = 0.5 * spec.L - (bh + 1) * comp_len
        half = float(spec.half_breadth(x))
        for d in range(nd):
            fore, aft = bh * nd + d, (bh + 1) * nd + d
            # the watertight bulkhead reaches the bulkhead deck; above it, the deck's own head
            crest = max(spec.bulkhead_top, min(deck_top(x, d) - 0.3, max(floors[d], spec.bulkhead_top)))
            add(fore, aft, WEIR, x, 0.0, crest, max(1.0, 0.2 * 2 * half), K_OVER, bh, True, monitor=bh)
            area, sill = rng.uniform(1.0, 3.0), rng.uniform(0.0, 1.0)
            add(fore, aft, ORIFICE, x, 0.0, max(floors[d], float(spec.bottom(x))) + sill + 1.0, area, K_DOOR, bh, False)
    for k in range(ncmp):
        xa = 0.5 * spec.L - (k + 1) * comp_len
        for d in range(nd - 1):
            for f in (0.25, 0.75):
                x = xa + f * comp_len
                yb = max(1.0, 0.45 * float(spec.half_breadth(x)))
                add(k * nd + d, k * nd + d + 1, ORIFICE, x, yb if f < 0.5 else -yb, floors[d + 1], rng.uniform(0.5, 4.0), K_DOWN, k, True)
        nt = spec.top_openings
        for j in range(nt):
            x = xa + (j + 0.5) / nt * comp_len
            add(-1, k * nd + nd - 1, WEIR, x, 0.0, float(spec.deck(x)), TOP_OPEN_SHARE * comp_len / nt, K_TOP, k, True)
    # extra hatches between the decks of the midship compartments (engine and boiler rooms)
    for j in range(spec.extra_hatches):
        k = ncmp // 2 - 1 + (j // 2) % 2
        d = j % (nd - 1)
        x = 0.5 * spec.L - (k + 0.5) * comp_len
        add(k * nd + d, k * nd + d + 1, ORIFICE, x, 0.0, floors[d + 1], rng.uniform(0.5, 4.0), K_DOWN, k, True)
    # breaches: below the waterline in the forward compartments (from the second), on alternating sides; the first
    # `breaches` share the total area and are open, the reserve ones aft of them are closed (a sweep may open them)
    w = rng.uniform(0.5, 1.5, size=spec.breaches)
    w = w / w.sum()
    for j in range(spec.breaches + spec.reserve_breaches):
        k = min(1 + j, ncmp - 1)
        x = 0.5 * spec.L - (k + rng.uniform(0.3, 0.7)) * comp_len
        z = spec.draft - rng.uniform(2.0, 4.0)
        z = max(z, float(spec.bottom(x)) + 0.5)
        d = max(dd for dd in range(nd) if floors[dd] <= z)
        side = -1.0 if j % 2 == 0 else 1.0
        area = float(spec.breach_area * w[j]) if j < spec.breaches else float(spec.breach_area / spec.breaches)
        add(-1, k * nd + d, ORIFICE, x, side * float(spec.half_breadth(x)), z, area, K_BREACH, j + 1, j < spec.breaches)
    C["n"] = len(C["a"])
    return C


def sim_document(spec, sim_id, ship_id, ship_hash, cols, nodes, segs, hyd, conns):
    V, T = hyd["V"], spec.draft
    ms = RHO * V
    kg = hyd["KB"] + hyd["BM"] - spec.gm
    g0 = [hyd["LCB"], 0.0, kg]
    zO = kg - T
    Lp, B = spec.L, spec.B
    mh0 = ms * 2.0
    ith0 = ms * (0.25 * Lp) ** 2 * 2.0
    iph0 = ms * (0.38 * B) ** 2 * 1.2
    kz = RHO * GRAV * hyd["Awp"]
    kth = RHO * GRAV * V * hyd["BML"]
    kph = RHO * GRAV * V * spec.gm
    body = {"ms": ms, "KG": kg, "g0": g0, "XO": hyd["LCB"], "YO": 0.0, "mh0": mh0, "Ith0": ith0, "Iph0": iph0,
            "cDz": 2 * 0.6 * math.sqrt(kz * mh0), "cDth": 2 * 0.6 * math.sqrt(kth * ith0), "cDph": 2 * 0.12 * math.sqrt(kph * iph0),
            "qz": 0.5 * RHO * Lp * B * 0.8, "qth": 0.25 * RHO * B * (Lp / 2) ** 4, "qph": 0.25 * RHO * Lp * (B / 2) ** 4}
    nn = nodes["n"]
    st, sc = nodes["segStart"], nodes["segCount"]
    level, cx, cy, cz = [], [], [], []
    for n in range(nn):
        idx = range(st[n], st[n] + sc[n])
        a = [segs["a"][j] for j in idx]
        xs = [cols["x"][segs["col"][j]] for j in idx]
        ys = [cols["y"][segs["col"][j]] for j in idx]
        level.append(min(a) - T)
        cx.append(sum(xs) / len(xs))
        cy.append(sum(ys) / len(ys))
        cz.append(min(a))
    state0 = {"t": 0.0, "zO": zO, "pitch": 0.0, "roll": 0.0, "vz": 0.0, "wth": 0.0, "wph": 0.0, "vol": [0.0] * nn, "level": level,
              "cx": cx, "cy": cy, "cz": cz}
    groups = {"n": nn, "nodeStart": list(range(nn)), "nodeCount": [1] * nn, "nodes": list(range(nn)), "mode": [0] * nn,
              "px": [0.0] * nn, "py": [0.0] * nn, "pz": [0.0] * nn, "margin": 0.05}
    nb = spec.n_comp - 1
    monitors = {"n": nb, "threshold": 0.05, "id": [f"over{b:02d}" for b in range(nb)],
                "label": [f"Water flows over bulkhead {b:02d}" for b in range(nb)]}
    xb = 0.5 * spec.L
    marks = {"n": 4, "id": ["bow", "foredeck", "midship", "stern"],
             "label": ["Bow deck edge under", "Foredeck at a quarter length under", "Deck edge amidships under", "Stern keel clear"],
             "x": [xb - 2.0, xb - 0.25 * spec.L, 0.0, -xb + 3.0], "y": [0.0, float(spec.half_breadth(xb - 0.25 * spec.L)), 0.5 * spec.B, 0.0],
             "z": [float(spec.deck(xb - 2.0)), float(spec.deck(xb - 0.25 * spec.L)), float(spec.deck(0.0)), float(spec.bottom(-xb + 3.0))],
             "when": [0, 0, 0, 1]}
    conns = dict(conns, kindNames=KIND_NAMES, typeNames=["orifice", "weir"])
    hashed = [
        ("groups.nodeStart", "i32", groups["nodeStart"]), ("groups.nodeCount", "i32", groups["nodeCount"]), ("groups.nodes", "i32", groups["nodes"]),
        ("groups.mode", "u8", groups["mode"]), ("groups.px", "f64", groups["px"]), ("groups.py", "f64", groups["py"]), ("groups.pz", "f64", groups["pz"]),
        ("connections.a", "i32", conns["a"]), ("connections.b", "i32", conns["b"]), ("connections.type", "u8", conns["type"]),
        ("connections.x", "f64", conns["x"]), ("connections.y", "f64", conns["y"]), ("connections.z", "f64", conns["z"]),
        ("connections.area", "f64", conns["area"]), ("connections.coef", "f64", conns["coef"]), ("connections.kind", "u8", conns["kind"]),
        ("connections.idx", "i32", conns["idx"]), ("connections.en", "u8", conns["en"]), ("connections.tOn", "f64", conns["tOn"]),
        ("connections.skipGroup", "i32", conns["skipGroup"]), ("connections.monitor", "i32", conns["monitor"]),
        ("marks.x", "f64", marks["x"]), ("marks.y", "f64", marks["y"]), ("marks.z", "f64", marks["z"]), ("marks.when", "u8", marks["when"]),
        ("state0.vol", "f64", state0["vol"]), ("state0.level", "f64", state0["level"]),
        ("state0.cx", "f64", state0["cx"]), ("state0.cy", "f64", state0["cy"]), ("state0.cz", "f64", state0["cz"]),
    ]
    return {
        "format": "sinksim.compiled-sim", "formatVersion": 1, "id": sim_id, "ship": ship_id, "shipHash": ship_hash,
        "meta": {"title": f"{ship_id}: {spec.breaches} breaches, {spec.breach_area:g} m2 in total", "generator": "sinksim_b200.hullgen"},
        "constants": {"rho": RHO, "g": GRAV},
        "scheme": {"dt": spec.dt},
        "groups": groups, "connections": conns, "monitors": monitors, "marks": marks,
        "founder": {"hullTopBelow": -0.5, "pitchAbsAbove": 1.2, "buoyancyBelow": 1, "minT": 10},
        "body": body,
        "readout": {"xFP": 0.5 * spec.L, "xAP": -0.5 * spec.L},
        "state0": state0,
        "hash": hash_arrays(hashed),
    }


def fleet_specs(n, seed=20261204, columns=(1000, 20000), length=(100.0, 300.0), spaces=(16, 256)):
    """n hull specs of a mixed fleet: column counts log-uniform over `columns` on a 5:1 (length:beam) grid, length
    uniform over `length` (m) with the liner's proportions (beam, depth, sheer, draft, bottom rise and breach area
    scaled by L / 269 m), compartments x decks between `spaces` (2-4 decks, at least two columns per compartment)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        cols = float(np.exp(rng.uniform(np.log(columns[0]), np.log(columns[1]))))
        ny = max(3, int(round(math.sqrt(cols / 5.0))))
        nx = max(10, int(round(cols / ny)))
        L = float(rng.uniform(*length))
        k = L / 269.0
        decks = int(rng.integers(2, 5))
        lo = max(2, -(-spaces[0] // decks))
        hi = max(lo, min(spaces[1] // decks, nx // 2))
        comps = int(rng.integers(lo, hi + 1))
        out.append(HullSpec(L=L, B=28.0 * k, depth=18.0 * k, sheer=4.0 * k, nx=nx, ny=ny, n_comp=comps, n_decks=decks, draft=10.5 * k,
                            gm=0.8 * k, end_rise=3.0 * k, breach_area=1.2 * k * k, bulkhead_top=13.5 * k, top_openings=3, breaches=min(6, comps - 1),
                            reserve_breaches=min(2, max(0, comps - 1 - min(6, comps - 1)))))
    return out


def generate(spec=None, seed=20261203, ship_id="liner269", sim_id=None):
    """(ship document, sim document) of a parametric liner."""
    spec = spec or HullSpec()
    rng = np.random.default_rng(seed)
    cols = build_columns(spec)
    nodes, segs = build_nodes(spec, cols)
    hyd = hydrostatics(cols, spec.draft)
    ship = ship_document(spec, ship_id, cols, nodes, segs, hyd)
    conns = build_connections(spec, cols, nodes, rng)
    sim = sim_document(spec, sim_id or ship_id + "-breached", ship_id, ship["hash"]["all"], cols, nodes, segs, hyd, conns)
    sim["meta"]["seed"] = seed
    ship["meta"]["seed"] = seed
    return ship, sim


def write(out_dir, spec=None, seed=20261203, ship_id="liner269"):
    """Writes <out_dir>/<ship_id>.ship.json and .sim.json; returns their paths. Each file is written under a name of
    this process's and then renamed, so processes writing the same hull at once (one per GPU) never read half a file."""
    ship, sim = generate(spec, seed, ship_id)
    os.makedirs(out_dir, exist_ok=True)
    paths = (os.path.join(out_dir, f"{ship_id}.ship.json"), os.path.join(out_dir, f"{ship_id}.sim.json"))
    for doc, p in zip((ship, sim), paths):
        tmp = f"{p}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(doc, f)
        os.replace(tmp, p)
    return paths


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m sinksim_b200.hullgen")
    ap.add_argument("--out", required=True)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--id", default="liner269")
    args = ap.parse_args(argv)
    for p in write(args.out, seed=args.seed, ship_id=args.id):
        print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
