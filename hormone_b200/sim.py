"""The host step loop: HORMONE's main program driving the GPU step.

``Simulation`` reproduces the sequence of src/main/hormone.f90:63-179 for
the explicit hydro/MHD (+hyperbolic gravity) path: set-up from parameters,
initial condition, the initial ``timestep``/``gravity`` calls, then per step
``timestep -> gravity -> hydro_step -> phidamp -> time += dt`` with the
reference's end and output-time logic.  Every array operation of the step
runs on the GPU through the C ABI; the host only sequences the calls.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

from . import capi, grid as gridmod, ic


class Simulation:
    def __init__(self, cfg: dict, prims: Optional[Dict[str, np.ndarray]] = None, grvphi=None, grvpsi=None,
                 cgrav_old: float = 0.0, precision: int = 0):
        self.cfg = cfg
        self.grid = gridmod.make_grid(cfg)
        if prims is None:
            prims = ic.make(cfg, self.grid)
        st = ic.to_state(cfg, prims)
        self.ctx = capi.Context(cfg, self.grid, precision=precision)
        self.ctx.upload(u=st["u"], prim=list(st["prim"]), grvphi=grvphi, grvpsi=grvpsi)
        self.time = 0.0
        self.tn = 0
        self.t_out = cfg["t_out"]
        self.t_end = cfg["t_end"]
        self.dt = 0.0
        self.ch = 0.0
        self.mag_glm = bool(cfg["mag_on"]) and cfg["dim"] > 1
        self.gravity = cfg["gravswitch"] == 3
        if self.gravity:
            self.ctx.set_gravity_clock(0.0, cgrav_old)
        # hormone.f90:107-113
        self.dt, self.ch = self.ctx.timestep(self.time, self.t_out, self.t_end)
        if self.gravity:
            self.ctx.gravity_step(self.time, self.dt, self.tn)

    def step(self) -> bool:
        """One pass of hormone.f90:126-172; returns True when the run ended."""
        self.dt, self.ch = self.ctx.timestep(self.time, self.t_out, self.t_end)
        if self.gravity:
            self.ctx.gravity_step(self.time, self.dt, self.tn)
        self.ctx.hydro_step()
        if self.mag_glm:
            self.ctx.phidamp()
        self.time = self.time + self.dt
        self.tn += 1
        c = self.cfg
        if c["endstyle"] == 1 and self.time >= self.t_end:
            return True
        if c["endstyle"] == 2 and self.tn >= c["tnlim"]:
            return True
        if c["outstyle"] == 1 and self.time >= self.t_out:
            self.t_out = self.t_out + c["dt_out"]
        return False

    def run(self, max_steps: int = 10 ** 9) -> bool:
        for _ in range(max_steps):
            if self.step():
                return True
        return False

    def run_device(self, max_steps: int = 10 ** 9) -> bool:
        """The same loop with device-resident time (hmn_run): no host round
        trip per step; valid when the only output is at t_end."""
        t, n = self.ctx.run(self.time, self.t_end, max_steps)
        self.time = t
        self.tn += n
        return self.time >= self.t_end

    def state(self, gravity: bool = False) -> Dict[str, np.ndarray]:
        return self.ctx.download(gravity=gravity)

    def close(self):
        self.ctx.close()
