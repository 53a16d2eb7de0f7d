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
