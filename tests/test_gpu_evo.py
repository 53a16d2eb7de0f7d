"""hmn_evo, the totals of evo_output (output.f90:147-275), against the same
sums formed on the host from the downloaded state: Cartesian MHD, Cartesian
and spherical self-gravity (bound mass, energy and angular momentum), an
axisymmetric cylindrical grid and a stretched mesh.  The device sums per
block and then over blocks, so the comparison allows rounding: each total
within 1e-12 of the sum of its terms' magnitudes."""
import numpy as np
import pytest

from hormone_b200 import grid as G
from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def host_dvol(cfg, grid):
    n = cfg["n"]
    crd = cfg.get("crdnt", 0)
    if crd == 2:
        return G.spherical_dvol(grid, n)
    d1, d2, d3 = (grid[a]["dxi"][2:n[a] + 2] for a in range(3))
    if crd == 1:
        xi = grid[0]["xi"]
        ar = xi[2:n[0] + 2] * xi[2:n[0] + 2] - xi[1:n[0] + 1] * xi[1:n[0] + 1]
        f4 = 4.0 if n[1] == 1 else 1.0
        return 0.5 * ar[None, None, :] * d2[None, :, None] * d3[:, None, None] * f4
    return d1[None, None, :] * d2[None, :, None] * d3[:, None, None]


def host_terms(cfg, grid, st, gravity):
    """The per-cell terms of each total (output.f90:163-233)."""
    n = cfg["n"]
    dv = host_dvol(cfg, grid)
    d, v1, v2, v3, e = st["d"], st["v1"], st["v2"], st["v3"], st["e"]
    b1, b2, b3 = st["b1"], st["b2"], st["b3"]
    eint = e - 0.5 * d * (v1 * v1 + v2 * v2 + v3 * v3) - 0.5 * (b1 * b1 + b2 * b2 + b3 * b3)
    x1 = grid[0]["x"][2:n[0] + 2][None, None, :]
    crd = cfg.get("crdnt", 0)
    if crd == 1:
        jl = d * x1 * v2 * dv
    elif crd == 2:
        jl = d * x1 * grid[1]["sinc"][2:n[1] + 2][None, :, None] * v3 * dv
    else:
        jl = np.zeros_like(d)
    t = {"Mtot": d * dv, "Etot": e * dv, "Eitot": eint * dv,
         "Ektot": 0.5 * d * (v1 * v1 + v2 * v2 + v3 * v3) * dv,
         "Ebtot": 0.5 * (b1 * b1 + b2 * b2 + b3 * b3) * dv, "Jtot": jl}
    if gravity:
        ph = st["grvphi"]
        bound = ph + (e - eint) / d <= 0.0
        t["Egtot"] = d * (ph - 0.5 * ph) * dv
        t["Mbound"] = np.where(bound, d * dv, 0.0)
        t["Ebound"] = np.where(bound, (e + d * (ph - 0.5 * ph)) * dv, 0.0)
        t["Jbound"] = np.where(bound, jl, 0.0)
    return t


def check(cfg, prims, steps, grvphi=None):
    gravity = cfg["gravswitch"] == 3
    sim = Simulation(cfg, prims, grvphi=grvphi)
    for _ in range(steps):
        sim.step()
    got = sim.ctx.evo()
    line = sim.evo()
    st = sim.state(gravity=gravity)
    sim.close()
    terms = host_terms(cfg, G.make_grid(cfg), st, gravity)
    for k, t in terms.items():
        tol = 1e-12 * float(np.sum(np.abs(t))) + 1e-300
        assert abs(got[k] - float(np.sum(t))) <= tol, (k, got[k], float(np.sum(t)))
    assert line["tn"] == steps and "Mtot" in line
    assert ("Egtot" in line) == gravity and ("Ebtot" in line) == bool(cfg["mag_on"])
    return got


def test_evo_cartesian_mhd():
    cfg, prims = cases.ot3d(16)
    got = check(cfg, prims, 3)
    assert got["Mtot"] > 0.0 and got["Ebtot"] > 0.0 and got["Jtot"] == 0.0


def test_evo_cartesian_self_gravity():
    cfg, prims, phi = cases.polytrope(16)
    got = check(cfg, prims, 3, grvphi=phi)
    assert got["Egtot"] < 0.0 and 0.0 < got["Mbound"] <= got["Mtot"]


def test_evo_spherical_self_gravity():
    cfg, prims, phi = cases.polytrope_spherical()
    check(cfg, prims, 3, grvphi=phi)


def test_evo_cylindrical_angular_momentum():
    cfg, prims = cases.cylindrical((24, 1, 18), mag=True)
    got = check(cfg, prims, 3)
    assert got["Jtot"] != 0.0


def test_evo_stretched_mesh():
    cfg, prims, phi = cases.polytrope_stretched(16)
    check(cfg, prims, 2, grvphi=phi)
