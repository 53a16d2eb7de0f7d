"""Initial conditions (host side), returned as primitive arrays.

Each function returns a dict of interior arrays with shape (nz, ny, nx)
(x fastest, as HORMONE's Fortran arrays are laid out) for d, p, v1..3,
b1..3 and phi.  The conversion to total energy is done by ``to_state``
exactly as src/main/initialcondition.f90:132-141 does it.

Transcendentals are evaluated with Python's ``math`` module (the C library,
one call per distinct argument) so that values match a Fortran build that
calls the same library.
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np

from .grid import centres

PI = math.acos(-1.0)  # src/main/modules.f90:86


def _zeros(cfg):
    n = cfg["n"]
    return np.zeros((n[2], n[1], n[0]), dtype=np.float64)


def _blank(cfg) -> Dict[str, np.ndarray]:
    return {k: _zeros(cfg) for k in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}


def shocktube(cfg, grid) -> Dict[str, np.ndarray]:
    """src/init/shocktube.f90:14-192 for sodshock_* and briowushock_*."""
    st = cfg["simtype"]
    direction = {"x": 0, "y": 1, "z": 2}[st[-1]]
    kind = st[:-2]
    dl, dr, pl, pr = 1.0, 0.125, 1.0, 0.1
    left = dict(v1=0.0, v2=0.0, v3=0.0, b1=0.0, b2=0.0, b3=0.0)
    right = dict(left)
    if kind == "briowushock":
        bvals = {0: ((0.75, 0.75), (1.0, -1.0), (0.0, 0.0)),
                 1: ((0.0, 0.0), (0.75, 0.75), (1.0, -1.0)),
                 2: ((1.0, -1.0), (0.0, 0.0), (0.75, 0.75))}[direction]
        for c in range(3):
            left[f"b{c + 1}"], right[f"b{c + 1}"] = bvals[c]
    elif kind != "sodshock":
        raise ValueError(f"unknown shock tube {st}")
    return riemann(cfg, direction, dict(d=dl, p=pl, **left), dict(d=dr, p=pr, **right))


def riemann(cfg, direction: int, left: dict, right: dict) -> Dict[str, np.ndarray]:
    """Two-state split along ``direction`` at index (is+ie)/2 (shocktube.f90:109-183)."""
    out = _blank(cfg)
    n = cfg["n"][direction]
    half = (1 + n) // 2  # Fortran (is_global+ie_global)/2 with is=1
    idx = np.arange(n)
    is_left = (idx + 1) <= half
    shape = [1, 1, 1]
    shape[2 - direction] = n
    mask = is_left.reshape(shape)
    for key in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3"):
        out[key] = np.where(mask, np.float64(left.get(key, 0.0)), np.float64(right.get(key, 0.0))) * np.ones_like(out[key])
    return out


def orszagtang(cfg, grid) -> Dict[str, np.ndarray]:
    """src/init/orszagtang.f90:14-80 (2-D planes xy, yz, xz)."""
    g = cfg["gamma"]
    n = cfg["n"]
    out = _blank(cfg)
    out["d"][:] = g * g / (4.0 * PI)
    out["p"][:] = g / (4.0 * PI)
    s4 = math.sqrt(4.0 * PI)
    if n[2] == 1:  # xy plane: (a, b) = (x, y)
        a_ax, b_ax, va, vb, ba, bb = 0, 1, "v1", "v2", "b1", "b2"
    elif n[1] == 1:  # xz plane
        a_ax, b_ax, va, vb, ba, bb = 0, 2, "v1", "v3", "b1", "b3"
    elif n[0] == 1:  # yz plane
        a_ax, b_ax, va, vb, ba, bb = 1, 2, "v2", "v3", "b2", "b3"
    else:
        raise ValueError("orszagtang needs a 2-D grid")
    xa, xb = centres(grid, a_ax), centres(grid, b_ax)
    sin2b = np.array([math.sin(2.0 * PI * v) for v in xb])
    sin2a = np.array([math.sin(2.0 * PI * v) for v in xa])
    sin4a = np.array([math.sin(4.0 * PI * v) for v in xa])
    va_1d = np.array([-s for s in sin2b])
    ba_1d = np.array([-s / s4 for s in sin2b])
    bb_1d = np.array([s / s4 for s in sin4a])

    def bcast(vec, ax):
        shape = [1, 1, 1]
        shape[2 - ax] = len(vec)
        return np.broadcast_to(vec.reshape(shape), out["d"].shape)

    out[va] = np.array(bcast(va_1d, b_ax))
    out[vb] = np.array(bcast(sin2a, a_ax))
    out[ba] = np.array(bcast(ba_1d, b_ax))
    out[bb] = np.array(bcast(bb_1d, a_ax))
    return out


def orszagtang3d(cfg, grid, seed: int = 20261203, amp: float = 1e-3) -> Dict[str, np.ndarray]:
    """3-D Orszag-Tang-type vortex (not in the reference, which refuses 3-D):
    the xy-plane fields of orszagtang.f90:29-41 on every z plane, plus seeded
    uniform noise of amplitude ``amp`` on vz and Bz."""
    g = cfg["gamma"]
    out = _blank(cfg)
    out["d"][:] = g * g / (4.0 * PI)
    out["p"][:] = g / (4.0 * PI)
    s4 = math.sqrt(4.0 * PI)
    x, y = centres(grid, 0), centres(grid, 1)
    sy = np.array([math.sin(2.0 * PI * v) for v in y])
    sx = np.array([math.sin(2.0 * PI * v) for v in x])
    s4x = np.array([math.sin(4.0 * PI * v) for v in x])
    out["v1"][:] = (-sy)[None, :, None]
    out["v2"][:] = sx[None, None, :]
    out["b1"][:] = np.array([-s / s4 for s in sy])[None, :, None]
    out["b2"][:] = np.array([s / s4 for s in s4x])[None, None, :]
    rng = np.random.Generator(np.random.PCG64(seed))
    out["v3"][:] = rng.uniform(-amp, amp, size=out["d"].shape)
    out["b3"][:] = rng.uniform(-amp, amp, size=out["d"].shape)
    return out


def kelvin_helmholtz(cfg, grid, rho_ratio: float, bx: float, width: float = 0.05, ptb: float = 0.01):
    """Periodic tanh shear layer (the batched Kelvin-Helmholtz benchmark boxes; the reference's own
    KHtests.f90 uses an exponential profile and passive scalars instead):
    vx = 0.5*tanh((|y|-0.25)/width), rho = 1 outside and ``rho_ratio`` inside
    the layer, p = 2.5, vy = ptb*sin(4 pi x), Bx = ``bx``."""
    out = _blank(cfg)
    x, y = centres(grid, 0), centres(grid, 1)
    t = np.array([math.tanh((abs(v) - 0.25) / width) for v in y])
    out["v1"][:] = (0.5 * t)[None, :, None]
    out["d"][:] = (1.0 + (rho_ratio - 1.0) * 0.5 * (1.0 - t))[None, :, None]
    out["v2"][:] = np.array([ptb * math.sin(4.0 * PI * v) for v in x])[None, None, :]
    out["p"][:] = 2.5
    out["b1"][:] = bx
    return out


def kh_instability(cfg, grid) -> Dict[str, np.ndarray]:
    """src/init/KHtests.f90:14-58: exponential shear layer at |y| = 1/4
    (width 0.025, densities 1 and 2, velocities +-0.5), vy = 0.01 sin(4 pi x),
    p = 2.5, and two passive scalars marking the two fluids.  Returns the
    primitives with 'spc' of shape (2, nz, ny, nx)."""
    out = _blank(cfg)
    rho1, rho2, vv1, vv2 = 1.0, 2.0, 0.5, -0.5
    rhom, vvm = 0.5 * (rho1 - rho2), 0.5 * (vv1 - vv2)
    ptb, width = 1e-2, 0.025
    x, y = centres(grid, 0), centres(grid, 1)
    v1 = np.empty(len(y))
    d = np.empty(len(y))
    outer = np.empty(len(y), dtype=bool)
    for j, yy in enumerate(y):
        if abs(yy) > 0.25:
            ex = math.exp((-abs(yy) + 0.25) / width)
            v1[j] = vv1 - vvm * ex
            d[j] = rho1 - rhom * ex
            outer[j] = True
        else:
            ex = math.exp((abs(yy) - 0.25) / width)
            v1[j] = vv2 + vvm * ex
            d[j] = rho2 + rhom * ex
            outer[j] = False
    out["v1"][:] = v1[None, :, None]
    out["d"][:] = d[None, :, None]
    out["v2"][:] = np.array([ptb * math.sin(4.0 * PI * v) for v in x])[None, None, :]
    out["p"][:] = 2.5
    spc = np.zeros((2,) + out["d"].shape)
    spc[0][:] = np.where(outer, 1.0, 0.0)[None, :, None]
    spc[1][:] = np.where(outer, 0.0, 1.0)[None, :, None]
    out["spc"] = spc
    return out


def polytrope_n1(cfg, grid, rho_floor: float = 1e-6):
    """n=1 polytrope of unit radius centred on the origin (G=1, K=2/pi).

    rho = sin(pi r)/(pi r) inside r<1 (at least ``rho_floor``) and
    ``rho_floor`` outside; p = K rho^2 + rho_floor*GM/max(r,1) with M = 4/pi,
    i.e. the interior polytrope plus the hydrostatic pressure of a
    constant-density atmosphere in the exterior potential (continuous at
    r=1).  The potential is the analytic one: phi = -(4/pi)(1+rho_poly)
    inside, -4/(pi r) outside (from phi + 2K rho = -GM/R).
    Returns (prims, grvphi)."""
    out = _blank(cfg)
    K = 2.0 / PI
    GM = 4.0 / PI
    x, y, z = centres(grid, 0), centres(grid, 1), centres(grid, 2)
    r = np.sqrt(x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2)
    inside = r < 1.0
    pr = np.where(inside & (r > 0.0), PI * r, 1.0)
    poly = np.where(inside, np.where(r > 0.0, np.sin(pr) / pr, 1.0), 0.0)
    rho = np.maximum(poly, rho_floor)
    out["d"][:] = rho
    out["p"][:] = K * poly * poly + rho_floor * GM / np.maximum(r, 1.0)
    rs = np.where(r > 0.0, r, 1.0)
    phi = np.where(inside, -GM * (1.0 + poly), -GM / rs)
    return out, phi


def polytrope_n1_spherical(cfg, grid, rho_floor: float = 1e-6):
    """The n=1 polytrope of ``polytrope_n1`` on a spherical polar grid
    centred on it: the same profiles of the radius x1 of each cell.
    Returns (prims, grvphi)."""
    out = _blank(cfg)
    K = 2.0 / PI
    GM = 4.0 / PI
    r = np.broadcast_to(centres(grid, 0)[None, None, :], out["d"].shape)
    inside = r < 1.0
    pr = np.where(inside & (r > 0.0), PI * r, 1.0)
    poly = np.where(inside, np.where(r > 0.0, np.sin(pr) / pr, 1.0), 0.0)
    out["d"][:] = np.maximum(poly, rho_floor)
    out["p"][:] = K * poly * poly + rho_floor * GM / np.maximum(r, 1.0)
    rs = np.where(r > 0.0, r, 1.0)
    phi = np.ascontiguousarray(np.where(inside, -GM * (1.0 + poly), -GM / rs))
    return out, phi


def sedov(cfg, grid, energy: float = 1.0, radius: float = 0.05, rho0: float = 1.0, p0: float = 1e-5):
    """Cartesian Sedov-type blast: ``energy`` spread evenly over the cells
    whose centres lie within ``radius`` of the box centre."""
    out = _blank(cfg)
    cs = [centres(grid, a) for a in range(3)]
    mids = [0.5 * (cfg["extent"][a][0] + cfg["extent"][a][1]) for a in range(3)]
    r2 = ((cs[0] - mids[0])[None, None, :] ** 2 + (cs[1] - mids[1])[None, :, None] ** 2
          + (cs[2] - mids[2])[:, None, None] ** 2)
    inside = r2 < radius * radius
    if not inside.any():
        inside = r2 == r2.min()
    dv = 1.0
    for a in range(3):
        dv *= grid[a]["dxi"][2]
    vol = inside.sum() * dv
    out["d"][:] = rho0
    out["p"][:] = np.where(inside, (cfg["gamma"] - 1.0) * energy / vol, p0)
    return out


def sedov_spherical(cfg, grid) -> Dict[str, np.ndarray]:
    """Spherical Sedov-Taylor blast of src/init/sedov.f90:14-64: density
    damb everywhere; the energy Eexp as pressure (gamma-1)*Eexp/vol_inj in
    the first ten radial cells (vol_inj their volume), and the ambient
    pressure 1e-3*Eexp/vol_tot elsewhere; at rest."""
    from .grid import fortran_sum, spherical_dvol

    out = _blank(cfg)
    i_inj = 10
    damb, eexp = float(cfg.get("damb", 1.0)), float(cfg.get("Eexp", 1.0))
    dvol = spherical_dvol(grid, cfg["n"])
    vol_inj = fortran_sum(dvol[:, :, :i_inj])
    ein = eexp / vol_inj
    pin = (cfg["gamma"] - 1.0) * ein  # eos_p, eostype 0 (eos.f90:254-256)
    vol_tot = fortran_sum(dvol)
    pamb = 1e-3 * eexp / vol_tot
    out["d"][:] = damb
    out["p"][:] = pamb
    out["p"][:, :, :i_inj] = pin
    return out


def to_state(cfg, prims: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """Total energy and conserved variables from the initial primitives.

    e = eint + (d*0.5)*|v|^2 + 0.5*|B|^2 with eint = p/(gamma-1)
    (initialcondition.f90:136-141, eos.f90:287-289); U as conserve.f90:13-50.
    Returns dict with 'prim' = (d, v1, v2, v3, e, b1, b2, b3, phi) stacked and
    'u' the nvar conserved planes.
    """
    g1 = cfg["gamma"] - 1.0
    d = prims["d"]
    v1, v2, v3 = prims["v1"], prims["v2"], prims["v3"]
    b1, b2, b3 = prims["b1"], prims["b2"], prims["b3"]
    eint = prims["p"] / g1
    vv = v1 * v1 + v2 * v2 + v3 * v3
    bb = b1 * b1 + b2 * b2 + b3 * b3
    e = eint + d * 0.5 * vv + 0.5 * bb
    prim = np.stack([d, v1, v2, v3, e, b1, b2, b3, prims["phi"]])
    u = [d, d * v1, d * v2, d * v3, e]
    if cfg["mag_on"]:
        u += [b1, b2, b3]
        if cfg["dim"] > 1:
            u.append(prims["phi"])
    out = {"prim": np.ascontiguousarray(prim), "u": np.ascontiguousarray(np.stack(u))}
    if cfg.get("nspc", 0):
        out["spc"] = np.ascontiguousarray(prims["spc"][:cfg["nspc"]])
    return out


def restart_state(cfg, fields: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """State after a restart from a dump (restart.f90 -> readbin.f90, then
    conserve.f90:13-50): the primitives d, v1..3, e (total energy), B, phi
    as the dump holds them, U rebuilt from them.  Returns the layout of
    ``to_state``."""
    d = fields["d"]
    v1, v2, v3, e = fields["v1"], fields["v2"], fields["v3"], fields["e"]
    z = np.zeros_like(d)
    b1, b2, b3 = (fields.get(k, z) for k in ("b1", "b2", "b3"))
    phi = fields.get("phi", z)
    prim = np.stack([d, v1, v2, v3, e, b1, b2, b3, phi])
    u = [d, d * v1, d * v2, d * v3, e]
    if cfg["mag_on"]:
        u += [b1, b2, b3]
        if cfg["dim"] > 1:
            u.append(phi)
    out = {"prim": np.ascontiguousarray(prim), "u": np.ascontiguousarray(np.stack(u))}
    if cfg.get("nspc", 0):
        out["spc"] = np.ascontiguousarray(np.moveaxis(fields["spc"], -1, 0)[:cfg["nspc"]])
    return out


def make(cfg, grid, **kw):
    st = cfg["simtype"]
    if st == "KHinstability":
        return kh_instability(cfg, grid)
    if st.startswith(("sodshock", "briowushock")):
        return shocktube(cfg, grid)
    if st.startswith("orszagtang"):
        return orszagtang(cfg, grid)
    if st == "sedov_default":
        return sedov_spherical(cfg, grid)
    raise ValueError(f"no initial condition for simtype {st}")
