"""Failure reporting without faulting the GPU: a state with negative
internal energy (the reference stops in internalenergy, eos.f90:833-839,
or error_flux, numflux.f90:579-593) makes the entry point return
HMN_ENEG_EINT with the cell, and the context stays usable."""
import numpy as np
import pytest

from hormone_b200 import capi, grid as G, ic
from hormone_b200.sim import Simulation
from oracle.oracle import Oracle

import cases

pytestmark = pytest.mark.gpu


def test_negative_internal_energy_is_reported_with_cell():
    cfg, prims = cases.ot3d(12)
    prims["p"][5, 4, 3] = -1e-3  # planted on the host: eint < 0 in one cell
    with pytest.raises(capi.HmnError) as ei:
        Simulation(cfg, prims)
    assert ei.value.code == capi.HMN_ENEG_EINT
    assert ei.value.cell == (3, 4, 5)
    # the oracle stops on the same cell
    o = Oracle(cfg)
    o.set_prims(prims)
    with pytest.raises(RuntimeError):
        o.start()
    # a fresh context on the same device still works
    cfg2, prims2 = cases.ot3d(12)
    s = Simulation(cfg2, prims2)
    s.step()
    s.close()


def test_bad_configuration_is_rejected():
    cfg, prims = cases.ot3d(8)
    bad = dict(cfg)
    bad["rktype"] = 4
    with pytest.raises(capi.HmnError) as ei:
        capi.Context(bad, G.make_grid(cfg))
    assert ei.value.code == capi.HMN_EBADCFG


def test_curvilinear_metric_outside_the_path_is_rejected():
    """hmn_set_metric returns HMN_EBADCFG for a cylindrical grid with a
    solved phi axis, for passive scalars on a spherical grid and for an
    unknown coordinate system; the host-side configuration refuses the
    same set-ups before any device call."""
    from hormone_b200 import config

    cfg, prims = cases.spherical((12, 8, 4), mag=False, xi1s=0.2)
    grid = G.make_grid(cfg)
    ctx = capi.Context(cfg, grid)  # spherical: accepted
    m = capi.HmnMetric()
    for code in (3, -1):
        assert capi.lib().hmn_set_metric(ctx.h, code, capi.ctypes.byref(m)) == capi.HMN_EBADCFG
    ctx.close()
    # a 3-D Cartesian context asked to become cylindrical (phi solved)
    cfg3, _ = cases.ot3d(8)
    ctx3 = capi.Context(cfg3, G.make_grid(cfg3))
    keep = [np.ones(12) for _ in range(3)]
    m.detg1, m.idetg1, m.sx1 = (capi._dp(a) for a in keep)
    assert capi.lib().hmn_set_metric(ctx3.h, 1, capi.ctypes.byref(m)) == capi.HMN_EBADCFG
    ctx3.close()
    with pytest.raises(ValueError):
        config.resolve("cyl", overrides=dict(ie=8, je=8, ke=8, crdnt=1))
    with pytest.raises(ValueError):
        config.resolve("sph", overrides=dict(ie=8, je=8, ke=8, crdnt=2, compswitch=2, spn=2))
    with pytest.raises(ValueError):
        config.resolve("sph", overrides=dict(ie=8, je=8, ke=8, crdnt=2, gravswitch=3, gbtype=0))
    with pytest.raises(ValueError):
        config.resolve("sph", overrides=dict(ie=8, je=1, ke=1, crdnt=2, gravswitch=3, gbtype=1))
