"""The sample sets of the reference's portable-math test (tests/test_portable_math.cpp:40-105 of the reference):
SplitMix64 seeded 20261008, the same draws in the same order, vectorised with numpy's wrapping uint64 arithmetic."""
import numpy as np

GOLDEN_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(seed, n):
    """The first n outputs of SplitMix64 from `seed` (state advanced before each output)."""
    with np.errstate(over="ignore"):
        s = np.uint64(seed) + GOLDEN_GAMMA * np.arange(1, n + 1, dtype=np.uint64)
        z = (s ^ (s >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform(bits):
    return (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def rng_range(bits, lo, hi):
    return lo + (hi - lo) * uniform(bits)


def reference_samples(n=400000):
    """(sin/cos arguments, pow (x, y), scalbn (x, n)) exactly as the reference test draws them."""
    # sin and cos: one draw per sample, four ranges in turn
    d = splitmix64(20261008, n)
    i = np.arange(n)
    ranges = [(-1.5, 1.5), (-3.0, 3.0), (-100.0, 100.0), (-8.0e5, 8.0e5)]
    trig = np.empty(n)
    for k, (lo, hi) in enumerate(ranges):
        trig[i % 4 == k] = rng_range(d[i % 4 == k], lo, hi)
    special = np.array([0.0, -0.0, 1e-30, -1e-30, 0.785398163397448279, 1.5707963267948966, 3.141592653589793, 1e-10, 1e300])
    trig = np.concatenate([trig, special])
    # pow: one draw for cases 0 and 1, two for the others, in sample order
    case = i % 6
    ndraw = np.where(case < 2, 1, 2)
    start = n + np.concatenate([[0], np.cumsum(ndraw)[:-1]])
    total = int(ndraw.sum())
    d = splitmix64(20261008, n + total + 2 * 20000)
    a = d[start]
    b = d[np.where(case < 2, start, start + 1)]
    x = np.empty(n)
    y = np.empty(n)
    m = case == 0; x[m] = uniform(a[m]); y[m] = 1.5
    m = case == 1; x[m] = uniform(a[m]); y[m] = 0.385
    m = case == 2; x[m] = rng_range(a[m], 1e-6, 1e3); y[m] = rng_range(b[m], -3.0, 3.0)
    m = case == 3; x[m] = rng_range(a[m], 0.5, 2.0); y[m] = rng_range(b[m], -200.0, 200.0)
    m = case == 4; x[m] = -rng_range(a[m], 0.1, 10.0); y[m] = np.trunc(rng_range(b[m], -6.0, 6.0))
    m = case == 5; x[m] = rng_range(a[m], 1e-300, 1e300); y[m] = rng_range(b[m], -1.0, 1.0)
    sx = np.array([0.0, -0.0, 1.0, -1.0, 2.0, 0.5, 1e-310, 1e308, -3.0])
    sy = np.array([0.0, 1.0, -1.0, 2.0, 0.5, 3.0, -2.0, 0.385, 1.5, 1e10, -1e10, 1024.0, -1075.0])
    px = np.concatenate([x, np.repeat(sx, len(sy))])
    py = np.concatenate([y, np.tile(sy, len(sx))])
    # scalbn: two draws per sample (x, then n)
    base = n + total
    k = np.arange(20000)
    bx = d[base + 2 * k]
    bn = d[base + 2 * k + 1]
    scx = rng_range(bx, -10.0, 10.0)
    scn = np.trunc(rng_range(bn, -1100.0, 1100.0))
    return trig, (px, py), (scx, scn)
