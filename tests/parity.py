"""Shared helpers for the parity tests: run the same IC through the oracle and the CUDA path."""
from __future__ import annotations

import numpy as np

from imogen_b200 import problems
from oracle import cpp_oracle

FIELDS = ("mass", "mom", "ener", "mag", "cellmag")


def rel_l1(a, b):
    """sum|a-b| / sum|b| (per variable), the north-star error measure."""
    den = np.sum(np.abs(b))
    num = np.sum(np.abs(a - b))
    return float(num / den) if den > 0 else float(num)


def errors(sa, sb):
    out = {}
    for k in FIELDS:
        a, b = np.asarray(sa[k]), np.asarray(sb[k])
        if a.ndim == 4:
            for c in range(3):
                out[f"{k}{'xyz'[c]}"] = rel_l1(a[c], b[c])
        else:
            out[k] = rel_l1(a, b)
    return out


def errors_vector(sa, sb):
    """rho and E per variable; momentum and B as vectors: sum|a-b| / sum|b| over all components
    (components that start at zero, like vz in a 2-D-seeded KH layer, are mostly round-off)."""
    out = {}
    for k in ("mass", "ener"):
        out[k] = rel_l1(np.asarray(sa[k]), np.asarray(sb[k]))
    for k in ("mom", "mag"):
        out[k] = rel_l1(np.asarray(sa[k]), np.asarray(sb[k]))
    return out


def smooth_state(grid, seed=0, mhd=True, gamma=5 / 3, amp=0.2):
    """A smooth, well-resolved random-phase state (positive density and pressure)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = grid
    x, y, z = np.meshgrid((np.arange(nx) + .5) / nx, (np.arange(ny) + .5) / ny, (np.arange(nz) + .5) / nz,
                          indexing="ij")
    ph = rng.uniform(0, 2 * np.pi, size=8)
    rho = 1 + amp * np.sin(2 * np.pi * x + ph[0]) * np.cos(2 * np.pi * y + ph[1]) + 0.02 * rng.random(grid)
    mom = np.stack([0.3 * np.sin(2 * np.pi * y + ph[2]), 0.2 * np.cos(2 * np.pi * x + ph[3] + z),
                    0.1 * np.sin(2 * np.pi * (x + y) + ph[4])]) * rho
    if mhd:
        mag = np.stack([0.2 * np.cos(2 * np.pi * y + ph[5]) + 0.05, 0.1 * np.sin(2 * np.pi * x + ph[6]),
                        0.05 * np.cos(2 * np.pi * (x - y) + ph[7])])
    else:
        mag = np.zeros((3,) + tuple(grid))
    P = 1 + 0.1 * np.cos(2 * np.pi * (x - y))
    ener = P / (gamma - 1) + 0.5 * (mom ** 2).sum(0) / rho + 0.5 * (mag ** 2).sum(0)
    return rho, mom, ener, mag


def make_pair(settings, state, precision="fp64"):
    """(oracle Sim, ImogenRun) constructed from the same settings and IC."""
    from imogen_b200 import ImogenRun
    o = cpp_oracle.Sim(**problems.oracle_kwargs(settings))
    o.set_state(*state)
    g = ImogenRun(precision=precision, **settings)
    g.set_state(*state)
    return o, g
