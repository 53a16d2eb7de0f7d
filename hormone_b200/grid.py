"""Uniform Cartesian grid arrays, built as HORMONE's gridset builds them.

Each axis holds six arrays over Fortran indices ``is-2 .. ie+2`` (stored at
offset +2, length n+4): cell centres ``x``, right faces ``xi``, centre
spacing ``dx``, cell widths ``dxi`` and their inverses ``idx``/``idxi``.
Centres and faces are running sums (src/main/gridset.f90:46-68), so their
rounding differs from ``xis + (i+1/2)*h``; the kernels read these arrays
rather than recomputing coordinates, which keeps them bit-compatible with the
reference.  With self-gravity on, the spacings are reset to the cell widths
and the ghost layers re-accumulated (gridset.f90:71-81).
"""
from __future__ import annotations

from typing import Dict, List

import numpy as np

AXIS_KEYS = ("x", "xi", "dx", "dxi", "idx", "idxi")


def uniform_axis(n: int, xis: float, xie: float, gravity: bool = False) -> Dict[str, np.ndarray]:
    L = n + 4
    x, xi, dx, dxi, idx, idxi = ([0.0] * L for _ in range(6))

    def at(i):  # Fortran-style index relative to is -> list slot
        return i + 2

    h = (xie - xis) / float(n)
    for i in range(-2, n + 2):
        dxi[at(i)] = h
    for i in range(-1, n + 2):
        dx[at(i)] = 0.5 * (dxi[at(i - 1)] + dxi[at(i)])
        idxi[at(i)] = 1.0 / dxi[at(i)]
        idx[at(i)] = 1.0 / dx[at(i)]
    x[at(-1)] = xis - dxi[at(-1)] * 0.5
    x[at(-2)] = x[at(-1)] - dx[at(-1)]
    xi[at(-1)] = xis
    xi[at(-2)] = xis - dxi[at(-1)]
    for i in range(0, n + 2):
        x[at(i)] = x[at(i - 1)] + dx[at(i)]
        xi[at(i)] = xi[at(i - 1)] + dxi[at(i)]
    if gravity:
        for i in range(-2, n + 2):
            dx[at(i)] = dxi[at(i)]
            idx[at(i)] = 1.0 / dx[at(i)]
            idxi[at(i)] = 1.0 / dxi[at(i)]
        for i in (-1, -2):
            xi[at(i)] = xi[at(i + 1)] - dxi[at(i)]
            x[at(i)] = x[at(i + 1)] - dx[at(i)]
        for i in (n, n + 1):
            xi[at(i)] = xi[at(i - 1)] + dxi[at(i)]
            x[at(i)] = x[at(i - 1)] + dx[at(i)]
    return {k: np.array(v, dtype=np.float64) for k, v in zip(AXIS_KEYS, (x, xi, dx, dxi, idx, idxi))}


def make_grid(cfg) -> List[Dict[str, np.ndarray]]:
    grav = int(cfg.get("gravswitch", 0)) != 0
    return [uniform_axis(cfg["n"][a], cfg["extent"][a][0], cfg["extent"][a][1], grav) for a in range(3)]


def centres(grid, a: int) -> np.ndarray:
    """Interior cell centres of axis a."""
    return grid[a]["x"][2:-2]
