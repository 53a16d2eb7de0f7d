"""Shared set-ups for the parity tests: small seeded configurations that the
oracle runs in seconds, covering every limiter, boundary code 0-3, 1-D/2-D/3-D
grids, hydro and MHD, and the hyperbolic-gravity source."""
import numpy as np

from hormone_b200 import config, grid as G, ic


def golden_case(name):
    flat = name.endswith("_flat")
    st = name[:-5] if flat else name
    cfg = config.resolve(st + " test", overrides={"flux_limiter": "flat"} if flat else None)
    return cfg, ic.make(cfg, G.make_grid(cfg))


def ot3d(n=16, limiter="modified_mc", courant=0.9, seed=20261203, rktype=3):
    cfg = config.resolve("ot3d", overrides=dict(ie=n, je=n, ke=n, mag_on=True, gamma=1.6666666666666667,
                                                 courant=courant, flux_limiter=limiter, t_end=0.5, dt_out=0.5,
                                                 rktype=rktype))
    return cfg, ic.orszagtang3d(cfg, G.make_grid(cfg), seed=seed)


def kh2d(n=32, ratio=2.0, bx=0.05, bc_y=0, limiter="modified_mc"):
    ov = dict(ie=n, je=n, ke=1, mag_on=True, gamma=1.6666666666666667, flux_limiter=limiter, t_end=2.0, dt_out=2.0,
              xi1s=-0.5, xi1e=0.5, xi2s=-0.5, xi2e=0.5)
    for tag in ("is", "os", "iv", "ov"):
        ov[f"bc2{tag}"] = bc_y
    cfg = config.resolve("kh", overrides=ov)
    return cfg, ic.kelvin_helmholtz(cfg, G.make_grid(cfg), ratio, bx)


def add_scalars(cfg, prims, seed=11):
    """Passive scalars that sum to one (what compswitch 2 carries): for two,
    a smooth seeded field and its complement; for more, seeded positive
    weights normalised per cell."""
    rng = np.random.default_rng(seed)
    shape = prims["d"].shape
    n = int(cfg.get("nspc", 2)) or 2
    prims = dict(prims)
    if n == 2:
        base = 0.5 + 0.4 * np.sin(np.arange(shape[2]) * 0.37)[None, None, :] * np.cos(np.arange(shape[1]) * 0.21)[None, :, None]
        x = np.clip(base + 0.05 * rng.uniform(-1, 1, size=shape), 0.0, 1.0)
        prims["spc"] = np.stack([x, 1.0 - x])
        return prims
    w = rng.uniform(0.1, 1.0, size=(n,) + shape)
    prims["spc"] = w / w.sum(axis=0)
    return prims


def blast3d(n=16, bc=2, mag=False, limiter="minmod", nspc=0):
    ov = dict(ie=n, je=n, ke=n, mag_on=mag, gamma=1.4, flux_limiter=limiter, t_end=0.2, dt_out=0.2, courant=0.4)
    if nspc:
        ov.update(compswitch=2, spn=nspc)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = bc
    cfg = config.resolve("blast", overrides=ov)
    prims = ic.sedov(cfg, G.make_grid(cfg), energy=1.0, radius=0.15, p0=0.05)
    if mag:
        prims["b1"][:] = 0.3
        prims["b3"][:] = -0.2
    if nspc:
        prims = add_scalars(cfg, prims)
    return cfg, prims


def riemann3d(n=(12, 10, 8), seed=7, bc=(3, 1, 0), nspc=0):
    rng = np.random.default_rng(seed)
    ov = dict(ie=n[0], je=n[1], ke=n[2], mag_on=True, gamma=1.4, t_end=0.1, dt_out=0.1, courant=0.8)
    if nspc:
        ov.update(compswitch=2, spn=nspc)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = bc[a - 1]
    cfg = config.resolve("riemann", overrides=ov)
    st = [dict(d=10 ** rng.uniform(-1, 0.5), p=10 ** rng.uniform(-1, 0.5), v1=rng.uniform(-1, 1),
               v2=rng.uniform(-1, 1), v3=rng.uniform(-1, 1), b1=rng.uniform(-1, 1), b2=rng.uniform(-1, 1),
               b3=rng.uniform(-1, 1)) for _ in range(2)]
    prims = ic.riemann(cfg, 0, st[0], st[1])
    # break the symmetry along y and z as well
    prims["d"] *= 1.0 + 0.1 * np.sin(np.arange(n[1]))[None, :, None] * np.cos(np.arange(n[2]))[:, None, None]
    if nspc:
        prims = add_scalars(cfg, prims)
    return cfg, prims


def polytrope(n=16):
    ov = dict(ie=n, je=n, ke=n, mag_on=False, gamma=2.0, gravswitch=3, G=1.0, courant=0.9,
              xi1s=-2.0, xi1e=2.0, xi2s=-2.0, xi2e=2.0, xi3s=-2.0, xi3e=2.0, t_end=1.0, dt_out=1.0)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = 3
    cfg = config.resolve("polytrope_cart", overrides=ov)
    prims, phi = ic.polytrope_n1(cfg, G.make_grid(cfg))
    return cfg, prims, phi


def polytrope_stretched(n=16, x3min=0.18):
    """The polytrope on a z mesh of geometrically growing widths
    (kmesh=1, utils.f90:351-404)."""
    ov = dict(ie=n, je=n, ke=n, mag_on=False, gamma=2.0, gravswitch=3, G=1.0, courant=0.9, kmesh=1, x3min=x3min,
              xi1s=-2.0, xi1e=2.0, xi2s=-2.0, xi2e=2.0, xi3s=-2.0, xi3e=2.0, t_end=1.0, dt_out=1.0)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = 3
    cfg = config.resolve("polytrope_cart", overrides=ov)
    prims, phi = ic.polytrope_n1(cfg, G.make_grid(cfg))
    return cfg, prims, phi


def cell_volumes(cfg, grid):
    """dvol of metric.f90 (norm weights of tests.f90)."""
    if cfg.get("crdnt", 0) == 2:
        return G.spherical_dvol(grid, cfg["n"])
    n = cfg["n"]
    return np.full((n[2], n[1], n[0]), grid[0]["dxi"][2] * grid[1]["dxi"][2] * grid[2]["dxi"][2])


def spherical(n=(24, 16, 1), mag=True, seed=5, xi1s=0.0, imesh=0, limiter="modified_mc", bc_r=(1, 2)):
    """A spherical polar grid (crdnt=2: r, theta, phi) holding a seeded,
    perturbed over-pressured core with small random velocities and a
    uniform field along the polar axis; the azimuthal components vanish on
    the axis like sin(theta)."""
    rng = np.random.default_rng(seed)
    ov = dict(ie=n[0], je=n[1], ke=n[2], crdnt=2, mag_on=mag, gamma=1.6666666666666667, xi1s=xi1s, xi1e=1.0,
              imesh=imesh, x1min=0.03, flux_limiter=limiter, t_end=1.0, dt_out=1.0, courant=0.8,
              bc1is=bc_r[0], bc1iv=bc_r[0], bc1os=bc_r[1], bc1ov=bc_r[1])
    cfg = config.resolve("spherical", overrides=ov)
    grid = G.make_grid(cfg)
    r = G.centres(grid, 0)[None, None, :]
    th = G.centres(grid, 1)[None, :, None]
    shape = (n[2], n[1], n[0])
    prims = {k: np.zeros(shape) for k in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}
    prims["d"][:] = 1.0 + 0.2 * rng.random(shape)
    prims["p"][:] = np.where(r < 0.3, 2.0, 0.5) * (1.0 + 0.1 * rng.random(shape))
    prims["v1"][:] = 0.1 * rng.uniform(-1.0, 1.0, shape)
    prims["v2"][:] = 0.1 * rng.uniform(-1.0, 1.0, shape)
    prims["v3"][:] = 0.1 * np.sin(th) * rng.uniform(-1.0, 1.0, shape)
    if mag:
        prims["b1"][:] = 0.2 * np.cos(th) + 0.02 * rng.uniform(-1.0, 1.0, shape)
        prims["b2"][:] = -0.2 * np.sin(th) + 0.02 * rng.uniform(-1.0, 1.0, shape)
        prims["b3"][:] = 0.02 * np.sin(th) * rng.uniform(-1.0, 1.0, shape)
    return cfg, prims


def polytrope_spherical(n=(24, 12, 8), xi1s=0.0, xi1e=2.0, imesh=0):
    """The n=1 polytrope on a spherical polar grid with hyperbolic
    self-gravity (Robin outer boundary, gbtype=1)."""
    ov = dict(ie=n[0], je=n[1], ke=n[2], crdnt=2, mag_on=False, gamma=2.0, gravswitch=3, gbtype=1, G=1.0,
              courant=0.9, xi1s=xi1s, xi1e=xi1e, imesh=imesh, x1min=0.02, t_end=1.0, dt_out=1.0,
              bc1is=1, bc1iv=1, bc1os=2, bc1ov=2)
    cfg = config.resolve("polytrope_sph", overrides=ov)
    prims, phi = ic.polytrope_n1_spherical(cfg, G.make_grid(cfg))
    return cfg, prims, phi


def cylindrical(n=(32, 1, 24), mag=True, seed=9, xi1s=0.0, imesh=0, kmesh=0, limiter="modified_mc"):
    """An axisymmetric cylindrical grid (crdnt=1: R, z with one phi cell)
    holding a seeded over-pressured core with small random velocities and a
    field along z plus a small toroidal part vanishing on the axis."""
    rng = np.random.default_rng(seed)
    ov = dict(ie=n[0], je=1, ke=n[2], crdnt=1, mag_on=mag, gamma=1.6666666666666667, xi1s=xi1s, xi1e=1.0,
              xi3s=-0.5, xi3e=0.5, imesh=imesh, x1min=0.03, kmesh=kmesh, x3min=0.04, flux_limiter=limiter,
              t_end=1.0, dt_out=1.0, courant=0.8, bc1is=1, bc1iv=1, bc1os=2, bc1ov=2,
              bc3is=0, bc3iv=0, bc3os=0, bc3ov=0)
    cfg = config.resolve("cylindrical", overrides=ov)
    grid = G.make_grid(cfg)
    r = G.centres(grid, 0)[None, None, :]
    z = G.centres(grid, 2)[:, None, None]
    shape = (n[2], 1, n[0])
    prims = {k: np.zeros(shape) for k in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}
    prims["d"][:] = 1.0 + 0.2 * rng.random(shape)
    prims["p"][:] = np.where(r * r + z * z < 0.09, 2.0, 0.5) * (1.0 + 0.1 * rng.random(shape))
    prims["v1"][:] = 0.1 * rng.uniform(-1.0, 1.0, shape)
    prims["v2"][:] = 0.1 * r * rng.uniform(-1.0, 1.0, shape)
    prims["v3"][:] = 0.1 * rng.uniform(-1.0, 1.0, shape)
    if mag:
        prims["b1"][:] = 0.02 * rng.uniform(-1.0, 1.0, shape)
        prims["b2"][:] = 0.05 * r * rng.uniform(-1.0, 1.0, shape)
        prims["b3"][:] = 0.2 + 0.02 * rng.uniform(-1.0, 1.0, shape)
    return cfg, prims


def wind_tunnel(n=(16, 12, 20), mag=False, nspc=0, seed=13):
    """A box fed through its inner x3 face by boundary code 10: a uniform
    wind (d, p, v3) enters with the flux of fluxboundary.f90:42-87, the
    ghosts below that face hold the wind state, the other faces are
    outgoing; a dense seeded clump sits in the flow.  Returns (cfg, prims,
    flux vector, Dirichlet ghost planes of the inner x3 face)."""
    rng = np.random.default_rng(seed)
    ov = dict(ie=n[0], je=n[1], ke=n[2], mag_on=mag, gamma=1.6666666666666667, t_end=1.0, dt_out=1.0, courant=0.8,
              xi1s=-0.5, xi1e=0.5, xi2s=-0.5, xi2e=0.5, xi3s=-0.5, xi3e=0.5)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = 2
    ov.update(bc3is=10, bc3iv=10)
    if nspc:
        ov.update(compswitch=2, spn=nspc)
    cfg = config.resolve("windtunnel", overrides=ov)
    grid = G.make_grid(cfg)
    x, y, z = (G.centres(grid, a) for a in range(3))
    r2 = x[None, None, :] ** 2 + y[None, :, None] ** 2 + z[:, None, None] ** 2
    shape = (n[2], n[1], n[0])
    dw, pw, vw = 1.0, 0.6, 0.8
    prims = {k: np.zeros(shape) for k in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}
    prims["d"][:] = np.where(r2 < 0.04, 10.0, dw) * (1.0 + 0.05 * rng.random(shape))
    prims["p"][:] = pw
    prims["v3"][:] = np.where(r2 < 0.04, 0.0, vw)
    if mag:
        prims["b1"][:] = 0.1
        prims["b3"][:] = 0.2
    gm1 = cfg["gamma"] - 1.0
    ew = pw / gm1 + 0.5 * dw * vw * vw
    flux = np.zeros(9 + nspc)
    flux[0] = dw * vw
    flux[3] = dw * vw * vw + pw
    flux[4] = (ew + pw) * vw
    if mag:  # the field is carried in by the wind (B x v along z)
        flux[4] = flux[4] + (0.1 * 0.1) * vw
        flux[5] = -0.1 * vw
    area = n[0] * n[1]
    ghosts = np.zeros((8 + nspc, 2, area))
    ghosts[0], ghosts[1], ghosts[4] = dw, pw, vw
    if mag:
        ghosts[5], ghosts[7] = 0.1, 0.2
    if nspc:
        prims = add_scalars(cfg, prims)
        flux[9 + nspc - 1] = flux[0]  # the wind is the last species (fluxboundary.f90:80-81)
        ghosts[8 + nspc - 1] = 1.0
    return cfg, prims, flux, ghosts
