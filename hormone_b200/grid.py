"""Grid arrays, built as HORMONE's gridset builds them: Cartesian axes
(uniform or geometrical-series meshes) and spherical polar axes (r, theta,
phi) with their metric factors.

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

import math
from decimal import Decimal, localcontext
from typing import Dict, List, Tuple

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


def quad_sin_cos(x: float) -> Tuple[float, float]:
    """sin and cos of a binary64 value, summed as Taylor series to 60
    digits and rounded once to binary64.  The reference takes them in quad
    precision and rounds to double (gridset.f90:376-382); both are the
    correctly rounded values except in double-rounding cases far rarer than
    any grid here."""
    with localcontext() as ctx:
        ctx.prec = 60
        t = Decimal(x)  # exact
        t2 = t * t
        s, c = Decimal(0), Decimal(0)
        ts, tc = t, Decimal(1)
        n = 0
        eps = Decimal(10) ** -58
        while abs(ts) > eps or abs(tc) > eps:
            s += ts
            c += tc
            ts = -ts * t2 / ((2 * n + 2) * (2 * n + 3))
            tc = -tc * t2 / ((2 * n + 1) * (2 * n + 2))
            n += 1
        return float(s), float(c)


def spherical_grid(cfg) -> List[Dict[str, np.ndarray]]:
    """Spherical polar axes (crdnt=2) as gridset.f90:294-423 builds them
    without gravity, and the 1-D metric factors of metric.f90:102-151.

    r runs over [xi1s, xi1e] (uniform, or a geometrical series with imesh=1)
    with volumetric cell centres; theta over [0, pi] ([0, pi/2] for one
    theta cell or eq_sym), uniform, with volumetric centres; phi over
    [-pi, pi], uniform (one cell stands for a quarter turn).  Extra keys:
    axis 0 ``detg`` (xi1**2), ``idetg`` and ``sx`` (over is-1..ie+1);
    axis 1 ``sini``/``cosi``/``sinc`` (js-2..je+2), ``scot`` and ``sisin``
    (js-1..je+1).  With self-gravity the two outer radial ghosts continue
    the last cell ratio (:331-343)."""
    n1, n2, n3 = (int(v) for v in cfg["n"])
    grav = int(cfg.get("gravswitch", 0)) != 0
    if 1 < n3 < 4:
        raise ValueError(f"Error from ke {n3}: a spherical grid needs one or at least four phi cells")
    if int(cfg.get("jmesh", 0)) != 0 or int(cfg.get("kmesh", 0)) != 0:
        raise ValueError("spherical grids take uniform theta and phi meshes (jmesh=kmesh=0) on this path")
    lo, hi = (float(v) for v in cfg["extent"][0])
    imesh = int(cfg.get("imesh", 0)) if n1 > 1 else 0
    if imesh == 0:
        widths = [(hi - lo) / float(n1)] * (n1 + 4)
    elif imesh == 1:
        widths = geometric_widths(n1, lo, hi, float(cfg["x1min"]))
    else:
        raise ValueError(f"imesh={imesh}: only uniform (0) and geometrical-series (1) meshes are on this path")
    r = axis_from_widths(widths, lo)
    x, xi, dx, idx, dxi, idxi = (r[k].tolist() for k in ("x", "xi", "dx", "idx", "dxi", "idxi"))
    for s in range(1, n1 + 4):  # Fortran is-1 .. ie+2 (:323-329)
        a, b = xi[s], xi[s - 1]
        x[s] = 0.75 * (a + b) * (a * a + b * b) / (a * a + a * b + b * b)
        if s == 2:
            x[1] = -x[2]
        dx[s] = x[s] - x[s - 1]
        idx[s] = 1.0 / dx[s]
    if grav:  # :331-343, the potential's grid being the hydro grid (gie = ie)
        for s in (n1 + 2, n1 + 3):
            dxi[s] = dxi[s - 1] * dxi[n1 + 1] / dxi[n1]
            idxi[s] = 1.0 / dxi[s]
            xi[s] = xi[s - 1] + dxi[s]
            a, b = xi[s], xi[s - 1]
            x[s] = 0.75 * (a + b) * (a * a + b * b) / (a * a + a * b + b * b)
            dx[s] = x[s] - x[s - 1]
            idx[s] = 1.0 / dx[s]
        dx[0] = dxi[0]
        idx = [1.0 / v for v in dx]
        idxi = [1.0 / v for v in dxi]
    r.update(x=np.array(x), xi=np.array(xi), dx=np.array(dx), idx=np.array(idx), dxi=np.array(dxi),
             idxi=np.array(idxi))

    pi = math.pi  # acos(-1d0)
    xi2e = pi * 0.5 if (n2 == 1 or bool(cfg.get("eq_sym", False))) else pi
    th = axis_from_widths([xi2e / float(1 if n2 == 1 else n2)] * (n2 + 4), 0.0)
    x, xi, dx, idx = (th[k].tolist() for k in ("x", "xi", "dx", "idx"))
    sc = [quad_sin_cos(v) for v in xi]
    si, ci = [v[0] for v in sc], [v[1] for v in sc]
    sinc = [quad_sin_cos(v)[0] for v in x]  # arithmetic centres, before the volumetric ones
    for s in range(1, n2 + 4):  # js-1 .. je+2 (:385-392)
        x[s] = (xi[s - 1] * ci[s - 1] - xi[s] * ci[s] + si[s] - si[s - 1]) / (ci[s - 1] - ci[s])
        if s == 2:
            x[1] = -x[2]
        dx[s] = x[s] - x[s - 1]
        idx[s] = 1.0 / dx[s]
    th.update(x=np.array(x), dx=np.array(dx), idx=np.array(idx))

    ketmp = 4 if n3 == 1 else n3
    ph = axis_from_widths([(pi - -pi) / float(ketmp)] * (n3 + 4), -pi)

    # metric.f90:102-151 (1-D factors; the 2-D/3-D ones are their products)
    xi, dxi = r["xi"].tolist(), r["dxi"].tolist()
    detg, idetg, sx = [0.0] * (n1 + 4), [0.0] * (n1 + 4), [0.0] * (n1 + 4)
    for s in range(1, n1 + 3):
        a, b = xi[s], xi[s - 1]
        detg[s] = a * a
        idetg[s] = 3.0 / (dxi[s] * (a * a + a * b + b * b))
        sx[s] = 1.5 * (a + b) / (a * a + a * b + b * b)
    scot, sisin = [0.0] * (n2 + 4), [0.0] * (n2 + 4)
    xi2 = th["xi"].tolist()
    for s in range(1, n2 + 3):
        scot[s] = (si[s] - si[s - 1]) / (ci[s - 1] - ci[s])
        sisin[s] = (xi2[s] - xi2[s - 1]) / (ci[s - 1] - ci[s])
    r.update(detg=np.array(detg), idetg=np.array(idetg), sx=np.array(sx))
    th.update(sini=np.array(si), cosi=np.array(ci), scot=np.array(scot), sinc=np.array(sinc),
              sisin=np.array(sisin))
    return [r, th, ph]


def cylindrical_grid(cfg) -> List[Dict[str, np.ndarray]]:
    """Cylindrical axes (crdnt=1: R, phi, z) with one phi cell, as
    gridset.f90:145-292 builds them without gravity: R uniform or a
    geometrical series with the volumetric centres
    sqrt((xi1(i-1)^2 + xi1(i)^2)/2) (the ghost below the first face
    mirrored), a quarter turn of phi, z uniform or a geometrical series; and
    the metric factors of metric.f90:53-100 on axis 0: ``detg`` (xi1),
    ``idetg`` (2/(xi1(i)^2-xi1(i-1)^2)) and ``sx`` (2/(xi1(i)+xi1(i-1)))."""
    n1, n2, n3 = (int(v) for v in cfg["n"])
    if n2 != 1:
        raise ValueError("cylindrical grids take one phi cell on this path")
    out = []
    for a, (mesh_key, min_key) in ((0, MESH_KEYS[0]), (2, MESH_KEYS[2])):
        n, (lo, hi) = cfg["n"][a], cfg["extent"][a]
        mesh = int(cfg.get(mesh_key, 0)) if n > 1 else 0
        if mesh == 0:
            widths = [(hi - lo) / float(n)] * (n + 4)
        elif mesh == 1:
            widths = geometric_widths(n, lo, hi, float(cfg[min_key]))
        else:
            raise ValueError(f"{mesh_key}={mesh}: only uniform (0) and geometrical-series (1) meshes are on this path")
        out.append(axis_from_widths(widths, lo))
    r, z = out
    x, xi, dx, idx = (r[k].tolist() for k in ("x", "xi", "dx", "idx"))
    for s in range(1, n1 + 4):  # Fortran is-1 .. ie+2 (:187-193)
        x[s] = math.sqrt((xi[s - 1] * xi[s - 1] + xi[s] * xi[s]) * 5e-1)
        if s == 1:
            x[s] = -x[s]
        dx[s] = x[s] - x[s - 1]
        idx[s] = 1.0 / dx[s]
    detg, idetg, sx = [0.0] * (n1 + 4), [0.0] * (n1 + 4), [0.0] * (n1 + 4)
    for s in range(1, n1 + 3):
        a, b = xi[s], xi[s - 1]
        detg[s] = a
        idetg[s] = 2.0 / (a * a - b * b)
        sx[s] = 2.0 / (a + b)
    r.update(x=np.array(x), dx=np.array(dx), idx=np.array(idx), detg=np.array(detg), idetg=np.array(idetg),
             sx=np.array(sx))
    ph = axis_from_widths([2.0 * math.pi / 4.0] * (n2 + 4), float(cfg["extent"][1][0]))
    return [r, ph, z]


def make_grid(cfg) -> List[Dict[str, np.ndarray]]:
    """The three axes of gridset.f90: uniform (mesh 0) or geometrical series
    (mesh 1, first cell x?min wide); cylindrical with crdnt=1, spherical
    polar with crdnt=2."""
    if int(cfg.get("crdnt", 0)) == 2:
        return spherical_grid(cfg)
    if int(cfg.get("crdnt", 0)) == 1:
        return cylindrical_grid(cfg)
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


def spherical_dvol(grid, n) -> np.ndarray:
    """Cell volumes dvol(i,j,k) of a spherical grid, (nz, ny, nx), in the
    operation order of metric.f90:122-123:
    (xi1(i)**3-xi1(i-1)**3)/3 * (cosi(j-1)-cosi(j)) * dxi3(k) * fac_j * fac_k."""
    n1, n2, n3 = (int(v) for v in n)
    xi = grid[0]["xi"]
    a, b = xi[2:n1 + 2], xi[1:n1 + 1]
    vr = (a * a * a - b * b * b) / 3.0
    ci = grid[1]["cosi"]
    cd = ci[1:n2 + 1] - ci[2:n2 + 2]
    dxi3 = grid[2]["dxi"][2:n3 + 2]
    fac_j = 2.0 if n2 == 1 else 1.0
    fac_k = 4.0 if n3 == 1 else 1.0
    return vr[None, None, :] * cd[None, :, None] * dxi3[:, None, None] * fac_j * fac_k


def fortran_sum(a: np.ndarray) -> float:
    """Fortran SUM of an array section: one running sum in storage order
    (i fastest), no reassociation."""
    t = 0.0
    for v in np.ascontiguousarray(a).reshape(-1).tolist():
        t = t + v
    return t
