"""GPU FP64 path vs the CPU oracle, step by step, bit for bit.

Every case starts both implementations from the same initial primitives and
compares dt and the full conserved and primitive state after every step.
The FP64 kernels keep the reference's operation order with no fused
multiply-adds, so the expected difference is exactly zero (-0 and +0 compare
equal); a stated per-step tolerance of 1e-12 relative is therefore met
with margin.
"""
import numpy as np
import pytest

from hormone_b200 import config, grid as G, ic
from hormone_b200.sim import Simulation
from oracle.oracle import Oracle

import cases

pytestmark = pytest.mark.gpu

PRIMS = ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")


def compare(o, s, where):
    st = s.state()
    ou = o.u()
    assert st["u"].shape == ou.shape
    for q in range(ou.shape[0]):
        bad = np.flatnonzero(st["u"][q] != ou[q])
        assert bad.size == 0, f"{where}: u[{q}] differs at {bad[:5]}: {st['u'][q].flat[bad[:3]]} vs {ou[q].flat[bad[:3]]}"
    for k in PRIMS:
        assert np.array_equal(st[k], o.get(k)), f"{where}: primitive {k} differs"
    for n in range(int(s.cfg.get("nspc", 0))):
        assert np.array_equal(st["spc"][n], o.get(f"spc{n}")), f"{where}: scalar {n} differs"


def run_pair(cfg, prims, nsteps, grvphi=None, cgrav_old=0.0, check_every=1, dirichlet=None, fluxbound=None):
    o = Oracle(cfg)
    for (axis, side), vals in (dirichlet or {}).items():
        o.set_dirichlet(axis, side, vals)
    if fluxbound is not None:
        o.set_flux_boundary(fluxbound)
    o.set_prims(prims)
    if grvphi is not None:
        o.set_gravity_state(grvphi, None, cgrav_old)
    o.start()
    s = Simulation(cfg, prims, grvphi=grvphi, cgrav_old=cgrav_old)
    for (axis, side), vals in (dirichlet or {}).items():
        s.ctx.set_dirichlet(axis, side, vals)
    if fluxbound is not None:
        s.ctx.set_flux_boundary(fluxbound)
    compare(o, s, "initial state")
    assert s.dt == o.scalars()["dt"] and s.ch == o.scalars()["ch"]
    for n in range(nsteps):
        end_o = o.step()
        end_s = s.step()
        sc = o.scalars()
        assert s.dt == sc["dt"], (n, s.dt, sc["dt"])
        assert s.time == sc["time"]
        if (n + 1) % check_every == 0 or end_o:
            compare(o, s, f"step {n + 1}")
        assert end_o == end_s
        if end_o:
            break
    if grvphi is not None:
        g = s.state(gravity=True)
        assert np.array_equal(g["grvphi"], o.get("grvphi"))
        assert np.array_equal(g["grvpsi"], o.get("grvpsi"))
    s.close()
    return o, s


@pytest.mark.parametrize("name", ["sodshock_x", "sodshock_y_flat", "briowushock_z", "briowushock_x_flat"])
def test_shocktubes_step_by_step(name):
    cfg, prims = cases.golden_case(name)
    run_pair(cfg, prims, 60)


@pytest.mark.parametrize("name", ["orszagtang_xy", "orszagtang_xz_flat", "orszagtang_yz"])
def test_orszag_tang_2d_step_by_step(name):
    cfg, prims = cases.golden_case(name)
    run_pair(cfg, prims, 25, check_every=5)


@pytest.mark.parametrize("limiter", ["modified_mc", "minmod", "flat"])
def test_orszag_tang_3d(limiter):
    cfg, prims = cases.ot3d(16, limiter=limiter)
    run_pair(cfg, prims, 6)


def test_orszag_tang_3d_ragged_tiles():
    cfg, prims = cases.ot3d(13)
    run_pair(cfg, prims, 4)


def test_march_z_chunks_and_ragged_columns():
    """MHD with GLM on a 3-D grid whose z extent splits into several march
    chunks (three here: 16, 16 and 8 planes) over ragged 16x8 column tiles
    (20 x 12 cells), with a state that varies along every axis and periodic,
    reflecting and outflow faces."""
    cfg, prims = cases.riemann3d(n=(20, 12, 40), bc=(0, 3, 1))
    run_pair(cfg, prims, 4)


def test_march_z_chunks_hydro():
    """The same chunking without magnetic fields (the march's hydro form),
    with outflow faces on every side."""
    ov = dict(ie=24, je=9, ke=36, mag_on=False, gamma=1.4, flux_limiter="modified_mc", t_end=0.2, dt_out=0.2,
              courant=0.4)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = 1
    cfg = config.resolve("blast", overrides=ov)
    prims = ic.sedov(cfg, G.make_grid(cfg), energy=1.0, radius=0.2, p0=0.05)
    run_pair(cfg, prims, 6)


@pytest.mark.parametrize("bc_y", [0, 1])
def test_kelvin_helmholtz_2d(bc_y):
    cfg, prims = cases.kh2d(40, bc_y=bc_y)
    run_pair(cfg, prims, 10)


@pytest.mark.parametrize("bc", [1, 2, 3])
def test_blast_3d_boundaries(bc):
    cfg, prims = cases.blast3d(14, bc=bc, mag=(bc == 2))
    run_pair(cfg, prims, 8)


def test_random_riemann_mixed_boundaries():
    cfg, prims = cases.riemann3d()
    run_pair(cfg, prims, 8)


def test_polytrope_hyperbolic_gravity():
    cfg, prims, phi = cases.polytrope(16)
    run_pair(cfg, prims, 5, grvphi=phi, cgrav_old=0.0)


@pytest.mark.parametrize("rktype", [1, 2])
def test_runge_kutta_orders(rktype):
    """rungekutta.f90's first- and second-order schemes (buffer roles and
    coefficients differ from SSP-RK3)."""
    cfg, prims = cases.ot3d(12, rktype=rktype, courant=0.4)
    run_pair(cfg, prims, 6)
    cfg, prims = cases.golden_case("briowushock_x")
    cfg = dict(cfg, rktype=rktype, courant=0.4)
    run_pair(cfg, prims, 30)


@pytest.mark.parametrize("make", [lambda: cases.ot3d(16), lambda: cases.blast3d(14, bc=1, mag=True),
                                  lambda: cases.riemann3d()])
def test_tma_staged_region_fp64(monkeypatch, make):
    """The stencil region staged by TMA bulk tensor copies (forced on for
    FP64; even x extents, ragged tiles, every boundary code) gives the
    oracle's bits."""
    monkeypatch.setenv("HMN_TMA", "1")
    cfg, prims = make()
    run_pair(cfg, prims, 4)


@pytest.mark.parametrize("make", [lambda: cases.golden_case("KHinstability"),
                                  lambda: cases.golden_case("KHinstability_flat"),
                                  lambda: cases.blast3d(14, bc=1, nspc=2),
                                  lambda: cases.riemann3d(nspc=2),
                                  lambda: cases.blast3d(14, bc=1, nspc=6),
                                  lambda: cases.riemann3d(nspc=8),
                                  lambda: cases.riemann3d(n=(20, 18, 1), bc=(3, 0, 3), nspc=5)])
def test_passive_scalars(make):
    """Passive scalars advected with the mass flux (numflux.f90:200-212,
    rungekutta.f90:61-86): 2-D KH with two (the reference's own test), and
    3-D and 2-D grids with 2 to 8 (the 8-scalar tiles) under reflective,
    free and periodic boundaries, MHD and hydro."""
    cfg, prims = make()
    run_pair(cfg, prims, 6)


def _edge_dirichlet(cfg, prims, axis, side, scale=1.0):
    """Ghost values of a code-9 face: the edge cells' state, density and
    pressure times `scale`, on both ghost layers."""
    p = {k: np.asarray(v) for k, v in prims.items()}
    idx = [slice(None)] * 3
    idx[2 - axis] = 0 if side == 0 else -1
    planes = [p["d"][tuple(idx)] * scale, p["p"][tuple(idx)] * scale] + \
             [p[k][tuple(idx)] for k in ("v1", "v2", "v3", "b1", "b2", "b3")]
    if cfg.get("nspc", 0):
        planes += [p["spc"][n][tuple(idx)] for n in range(cfg["nspc"])]
    return np.ascontiguousarray(np.stack([np.stack([pl, pl]) for pl in planes]))


@pytest.mark.parametrize("nspc", [0, 2])
def test_linear_and_dirichlet_boundaries(nspc):
    """Codes 4 and 5 (linear extrapolation; with outflow-only normal
    velocity) and 9 (Dirichlet ghost values from the host) on every axis,
    against the oracle, with and without passive scalars."""
    from hormone_b200 import config, grid as G, ic

    ov = dict(ie=12, je=10, ke=8, mag_on=True, gamma=1.4, t_end=0.1, dt_out=0.1, courant=0.6,
              bc1is=3, bc1iv=3, bc1os=4, bc1ov=4, bc2is=5, bc2iv=5, bc2os=9, bc2ov=9,
              bc3is=4, bc3iv=5, bc3os=9, bc3ov=4)
    if nspc:
        ov.update(compswitch=2, spn=nspc)
    cfg = config.resolve("riemann", overrides=ov)
    rng = np.random.default_rng(5)
    st = [dict(d=10 ** rng.uniform(-0.5, 0.3), p=10 ** rng.uniform(-0.5, 0.3), v1=rng.uniform(-0.5, 0.5),
               v2=rng.uniform(-0.5, 0.5), v3=rng.uniform(-0.5, 0.5), b1=0.3, b2=rng.uniform(-0.5, 0.5),
               b3=rng.uniform(-0.5, 0.5)) for _ in range(2)]
    prims = ic.riemann(cfg, 0, st[0], st[1])
    prims["d"] *= 1.0 + 0.1 * np.sin(np.arange(10))[None, :, None] * np.cos(np.arange(8))[:, None, None]
    if nspc:
        prims = cases.add_scalars(cfg, prims)
    dirichlet = {(1, 1): _edge_dirichlet(cfg, prims, 1, 1, 1.05), (2, 1): _edge_dirichlet(cfg, prims, 2, 1, 0.95)}
    run_pair(cfg, prims, 8, dirichlet=dirichlet)


def test_geometric_series_mesh():
    """Stretched cells on two axes (imesh=jmesh=1): the modified-MC factors,
    face offsets and divergence widths that vary per cell."""
    from hormone_b200 import config, grid as G, ic

    cfg = config.resolve("kh", overrides=dict(ie=40, je=32, ke=1, mag_on=True, gamma=1.6666666666666667,
                                              imesh=1, x1min=0.015, jmesh=1, x2min=0.02, t_end=2.0, dt_out=2.0,
                                              xi1s=-0.5, xi1e=0.5, xi2s=-0.5, xi2e=0.5,
                                              bc2is=3, bc2os=3, bc2iv=3, bc2ov=3))
    prims = ic.kelvin_helmholtz(cfg, G.make_grid(cfg), 2.0, 0.05)
    run_pair(cfg, prims, 10)


@pytest.mark.parametrize("make", [lambda: cases.spherical((40, 1, 1), mag=True),
                                  lambda: cases.spherical((24, 16, 1), mag=True),
                                  lambda: cases.spherical((16, 12, 8), mag=False),
                                  lambda: cases.spherical((20, 1, 8), mag=True, xi1s=0.1, imesh=1, bc_r=(3, 3)),
                                  lambda: cases.spherical((21, 10, 4), mag=True, xi1s=0.2, limiter="minmod")],
                         ids=["radial-mhd", "r-theta-mhd", "r-theta-phi", "r-phi-stretched", "shell-3d-minmod"])
def test_spherical_coordinates(make):
    """crdnt=2: metric-weighted flux divergence (rungekutta.f90:42-53),
    geometric source terms (source.f90:113-143) and the spherical CFL
    (timestep.f90:175-178 with metric.f90:117-130), bitwise vs the oracle."""
    cfg, prims = make()
    run_pair(cfg, prims, 12)


@pytest.mark.parametrize("n,xi1s", [((24, 12, 8), 0.0), ((20, 16, 1), 0.1), ((16, 8, 8), 0.2)],
                         ids=["3d-from-origin", "r-theta-shell", "3d-shell"])
def test_spherical_self_gravity(n, xi1s):
    """Hyperbolic self-gravity on spherical grids: the Laplacian of
    setup_grv_hyperbolic (axisymmetric and 3-D, Robin outer radius, the
    inner-radius term of a shell and its ghost held through the
    sub-cycles), the spherical gravity source terms and dtg_unit, bitwise
    against the oracle with the potential compared at the end."""
    cfg, prims, phi = cases.polytrope_spherical(n, xi1s=xi1s)
    run_pair(cfg, prims, 8, grvphi=phi)


@pytest.mark.parametrize("make", [lambda: cases.cylindrical((32, 1, 24), mag=True),
                                  lambda: cases.cylindrical((40, 1, 1), mag=True),
                                  lambda: cases.cylindrical((24, 1, 20), mag=False, xi1s=0.1, imesh=1, kmesh=1),
                                  lambda: cases.cylindrical((30, 1, 16), mag=True, xi1s=0.2, limiter="minmod")],
                         ids=["r-z-mhd", "radial-mhd", "r-z-stretched-shell", "r-z-minmod"])
def test_cylindrical_coordinates(make):
    """crdnt=1 with one phi cell: the xi1-weighted radial divergence
    (rungekutta.f90:42-53 with metric.f90:53-100), the cylindrical source
    terms (source.f90:88-111) and CFL, bitwise vs the oracle."""
    cfg, prims = make()
    run_pair(cfg, prims, 12)


@pytest.mark.parametrize("mag,nspc", [(False, 0), (True, 0), (False, 2)], ids=["hydro", "mhd", "two-species"])
def test_flux_boundary_code_10(mag, nspc):
    """Boundary code 10 at the inner x3 face: the host's wind flux replaces
    the Riemann flux there (numflux.f90:566, fluxboundary.f90:42-87) and the
    ghosts keep the host's values, bitwise vs the oracle."""
    cfg, prims, flux, ghosts = cases.wind_tunnel(mag=mag, nspc=nspc)
    run_pair(cfg, prims, 12, dirichlet={(2, 0): ghosts.reshape(-1)}, fluxbound=flux)
