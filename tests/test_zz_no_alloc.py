"""hmn_timestep_noalloc: the CFL timestep for callers that cannot allocate.

A host program whose device memory belongs to another runtime's pool, or one
that forbids allocation after start-up, cannot create an hmn_ctx (creation
allocates).  hmn_timestep_noalloc gives such callers the timestep from a
conserved state they already hold on the device, writing dt, ch and a status
into their own device memory; its only scratch is a static device array.

This file is collected last so that, if it fails, a run stopping at the
first failure has already run every other test.  It checks the result against
hmn_timestep (the allocating entry point) bit for bit, on two calls in a row
(the second sees the state one step later and reuses the same scratch), and
that oversize grids, ghosted layouts and negative-energy states are reported."""
import ctypes

import numpy as np
import pytest

from hormone_b200 import capi, config, grid as G
from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_timestep_matches_hmn_timestep_on_two_calls():
    import torch

    cfg, prims = cases.ot3d(24)
    sim = Simulation(cfg, prims)
    sim.step()  # from here on the primitives derive from U, as the no-alloc entry point derives them
    L = capi.lib()
    gs, keep = capi.grid_struct(cfg, sim.grid)
    ps = capi.params_struct(cfg)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        u = sim.state()["u"]
        u_dev = torch.from_numpy(np.ascontiguousarray(u)).cuda()
        dt_ref, ch_ref = sim.ctx.timestep(sim.time, sim.t_out, sim.t_end)
        out.fill_(-7.0)
        rc = L.hmn_timestep_noalloc(ctypes.byref(gs), ctypes.byref(ps), _ptr(u_dev), sim.time, sim.t_out, sim.t_end,
                                    _ptr(out), ctypes.c_void_p(stream.cuda_stream))
        assert rc == capi.HMN_OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[2] == 0.0, got
        assert got[0] == dt_ref, (call, got[0], dt_ref)
        assert got[1] == ch_ref, (call, got[1], ch_ref)
        sim.step()
    sim.close()


def test_noalloc_reports_negative_energy_and_rejects_oversize_grids():
    import torch

    cfg, prims = cases.ot3d(12)
    sim = Simulation(cfg, prims)
    sim.step()
    u = sim.state()["u"].copy()
    sim.close()
    u[4, 3, 2, 1] = -1.0  # total energy below zero in one cell, planted on the host
    L = capi.lib()
    gs, keep = capi.grid_struct(cfg, G.make_grid(cfg))
    ps = capi.params_struct(cfg)
    u_dev = torch.from_numpy(u).cuda()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.hmn_timestep_noalloc(ctypes.byref(gs), ctypes.byref(ps), _ptr(u_dev), 0.0, 1.0, 1.0, _ptr(out),
                                ctypes.c_void_p(stream.cuda_stream))
    assert rc == capi.HMN_OK
    torch.cuda.synchronize()
    assert out[2].item() == capi.HMN_ENEG_EINT
    big = config.resolve("big", overrides=dict(ie=5000, je=1, ke=1, t_end=1.0, dt_out=1.0))
    gb, keepb = capi.grid_struct(big, G.make_grid(big))
    rc = L.hmn_timestep_noalloc(ctypes.byref(gb), ctypes.byref(capi.params_struct(big)), _ptr(u_dev), 0.0, 1.0, 1.0,
                                _ptr(out), ctypes.c_void_p(stream.cuda_stream))
    assert rc == capi.HMN_EINVAL
    gg, keepg = capi.grid_struct(cfg, G.make_grid(cfg))
    gg.ghost = 2  # the state is read as packed planes; a ghosted layout is refused
    rc = L.hmn_timestep_noalloc(ctypes.byref(gg), ctypes.byref(ps), _ptr(u_dev), 0.0, 1.0, 1.0, _ptr(out),
                                ctypes.c_void_p(stream.cuda_stream))
    assert rc == capi.HMN_EINVAL
