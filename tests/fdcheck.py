"""Central differences of the trajectory objective on the C restatement, with the branch digest that tells whether the
stencil stayed on one branch path, beside the adjoint's gradient (the product's reverse step run on the host).
Test infrastructure for tests/test_adjoint_fd.py and for the stated agreement between the adjoint and finite differences.
"""
import math

import numpy as np

from _support import Oracle, adjoint_host_gradient


def objective_run(ship, sim, areas, steps, samples, trim_t, heave_t, digest=False):
    """J of one run with the given {connection: area}, and the run's branch digest."""
    o = Oracle(ship, sim, False)
    for c, a in areas.items():
        o.set_connection(int(c), area=float(a))
    if digest:
        o.digest_start()
    J, done = 0.0, 0
    for k, s in enumerate(samples):
        o.step(s - done)
        done = s
        r = o.readouts()
        trim, heave = r[1], 0.5 * (r[5] + r[6])
        J += (trim - trim_t[k]) ** 2 + (heave - heave_t[k]) ** 2
    if done < steps:
        o.step(steps - done)
    return J, (o.digest() if digest else None)


def chain_to_theta(space, theta, grad_area):
    """d J / d theta from d J / d area (the parameter space's map: kind log scales, then absolute areas)."""
    areas = space.areas(theta)
    g = np.zeros(space.dim)
    over = set(space.conns)
    for k, members in enumerate(space.members):
        g[k] = sum(grad_area[c] * areas[c] for c in members if c not in over)
    for j, c in enumerate(space.conns):
        g[len(space.kinds) + j] = grad_area[c]
    return g


def fd_versus_adjoint(ship, sim, space, theta, steps, samples, trim_t, heave_t, h_rel=1e-6):
    """Per parameter: (same branch path on both sides, central difference, adjoint). The step is h_rel x max(|theta_i|, 1)."""
    areas = space.areas(theta)
    en = np.array(sim["en"], dtype=np.uint8)
    area = np.array(sim["area"], dtype=np.float64)
    for c, a in areas.items():
        area[c] = a
    t_on = np.array(sim["tOn"], dtype=np.float64)
    J, ga, err = adjoint_host_gradient(ship, sim, en, area, t_on, steps, samples, trim_t, heave_t)
    if err:
        raise RuntimeError(f"adjoint error bits {err}")
    g = chain_to_theta(space, theta, ga)
    _, d0 = objective_run(ship, sim, areas, steps, samples, trim_t, heave_t, digest=True)
    out = []
    for i in range(space.dim):
        h = h_rel * max(abs(theta[i]), 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        jp, dp = objective_run(ship, sim, space.areas(tp), steps, samples, trim_t, heave_t, digest=True)
        jm, dm = objective_run(ship, sim, space.areas(tm), steps, samples, trim_t, heave_t, digest=True)
        fd = (jp - jm) / ((theta[i] + h) - (theta[i] - h))
        out.append((dp == d0 == dm, fd, g[i]))
    return J, out
