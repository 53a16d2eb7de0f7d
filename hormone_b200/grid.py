"""Cartesian grid arrays, built as HORMONE's gridset builds them (uniform
or geometrical-series meshes).

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


def geometric_widths(n: int, xis: float, xie: float, xmin: float) -> List[float]:
    """Cell widths of a geometrical-series mesh (imesh=1), restating
    src/main/utils.f90:351-404: the ratio xr solves
    (xr-1)*(xie-xis) = xmin*(xr**n-1) by Newton's method from 1.01; the first
    cell is xmin wide and each next one xr times wider.  Returns the n+4
    widths of indices is-2 .. ie+2."""
    xrmax, maxerr = 1.05, 1e-10
    xr = 1.01
    xrng, irng = xie - xis, float(n)
    if xrng / irng < xmin:
        raise ValueError("geometrical_series: xmin should be smaller or uniform mesh should be chosen")
    for _ in range(10000000):
        fx = (xr - 1.0) * xrng - xmin * (xr ** irng - 1.0)
        dfx = xrng - irng * xmin * xr ** (irng - 1.0)
        xrnew = xr - fx / dfx
        if abs((xrnew - xr) / xr) < maxerr:
            xr = xrnew
            break
        if xrnew < 1.0:
            xrnew = 2.0
        xr = xrnew
    if xr > xrmax:
        raise ValueError(f"geometrical_series: xmin too small ({xmin}, ratio {xr})")
    dxi = [0.0] * (n + 4)
    dxi[2] = xmin
    for i in range(1, n):
        dxi[i + 2] = dxi[i + 1] * xr
    dxi[1] = dxi[2]
    dxi[0] = dxi[3]
    dxi[n + 2] = dxi[n + 1] * xr
    dxi[n + 3] = dxi[n + 1] * xr * xr
    if xr - 1.0 < maxerr:
        dxi = [xrng / irng] * (n + 4)
    return dxi


def uniform_axis(n: int, xis: float, xie: float, gravity: bool = False) -> Dict[str, np.ndarray]:
    return axis_from_widths([(xie - xis) / float(n)] * (n + 4), xis, gravity)


def axis_from_widths(widths, xis: float, gravity: bool = False) -> Dict[str, np.ndarray]:
    """Centres, faces and spacings from the cell widths of indices is-2 ..
    ie+2 (gridset.f90:46-81, the same for every Cartesian mesh kind)."""
    L = len(widths)
    n = L - 4
    x, xi, dx, dxi, idx, idxi = ([0.0] * L for _ in range(6))

    def at(i):  # Fortran-style index relative to is -> list slot
        return i + 2

    for i in range(-2, n + 2):
        dxi[at(i)] = float(widths[at(i)])
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


MESH_KEYS = (("imesh", "x1min"), ("jmesh", "x2min"), ("kmesh", "x3min"))


def make_grid(cfg) -> List[Dict[str, np.ndarray]]:
    """The three axes of gridset.f90: uniform (mesh 0) or geometrical series
    (mesh 1, first cell x?min wide)."""
    grav = int(cfg.get("gravswitch", 0)) != 0
    out = []
    for a in range(3):
        n, (lo, hi) = cfg["n"][a], cfg["extent"][a]
        mesh_key, min_key = MESH_KEYS[a]
        mesh = int(cfg.get(mesh_key, 0)) if n > 1 else 0
        if mesh == 0:
            out.append(uniform_axis(n, lo, hi, grav))
        elif mesh == 1:
            out.append(axis_from_widths(geometric_widths(n, lo, hi, float(cfg[min_key])), lo, grav))
        else:
            raise ValueError(f"{mesh_key}={mesh}: only uniform (0) and geometrical-series (1) meshes are on this path")
    return out


def centres(grid, a: int) -> np.ndarray:
    """Interior cell centres of axis a."""
    return grid[a]["x"][2:-2]
