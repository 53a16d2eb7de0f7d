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

from . import binio, capi, grid as gridmod, ic


class Simulation:
    def __init__(self, cfg: dict, prims: Optional[Dict[str, np.ndarray]] = None, grvphi=None, grvpsi=None,
                 cgrav_old: float = 0.0, precision: int = 0, _state=None, _clock=None):
        self.cfg = cfg
        self.grid = gridmod.make_grid(cfg)
        if _state is None:
            if prims is None:
                prims = ic.make(cfg, self.grid)
            _state = ic.to_state(cfg, prims)
        st = _state
        self.ctx = capi.Context(cfg, self.grid, precision=precision)
        self.ctx.upload(u=st["u"], prim=list(st["prim"]), grvphi=grvphi, grvpsi=grvpsi)
        self.nspc = int(cfg.get("nspc", 0))
        if self.nspc:
            self.ctx.upload_scalars(st["spc"])
        self.time, self.tn = (0.0, 0) if _clock is None else _clock
        # restart.f90: t_out = time + dt_out after a restart
        self.t_out = cfg["t_out"] if _clock is None else self.time + cfg["dt_out"]
        self.t_end = cfg["t_end"]
        self.dt = 0.0
        self.ch = 0.0
        self.mag_glm = bool(cfg["mag_on"]) and cfg["dim"] > 1
        self.gravity = cfg["gravswitch"] == 3
        if self.gravity:
            self.ctx.set_gravity_clock(self.time, cgrav_old)
        # hormone.f90:107-113 (gravity only at tn == 0)
        self.dt, self.ch = self.ctx.timestep(self.time, self.t_out, self.t_end)
        if self.gravity and self.tn == 0:
            self.ctx.gravity_step(self.time, self.dt, self.tn)

    # -- checkpoints: output.f90:697-795 (write_bin) / restart.f90 -------------
    def checkpoint_begin(self, exact: bool = False):
        """Snapshot the current state on the device and copy it to the host
        in the background; the steps that follow run meanwhile.  exact=True
        also keeps the conserved planes, for a bit-exact resume."""
        arrays = self.ctx.checkpoint_begin(u=exact, gravity=self.gravity)
        cgrav_old = self.ctx.gravity_clock()[1] if self.gravity else 0.0
        self._ck = (self.tn, self.time, cgrav_old)
        return arrays

    def checkpoint_finish(self, path: Optional[str] = None) -> Dict[str, object]:
        """Wait for the snapshot; with a path, write it as a HORMONE dump
        (and, for an exact checkpoint, the conserved planes beside it as
        <path>.u.npy).  Returns the snapshot's fields, tn and time."""
        fields = self.ctx.checkpoint_wait()
        tn, time, cgrav_old = self._ck
        if path:
            binio.writebin(path, tn, time, fields, bool(self.cfg["mag_on"]), self.cfg["gravswitch"], cgrav_old,
                           species=self.cfg.get("species"))
            if "u" in fields:
                np.save(path + ".u.npy", fields["u"])
        out = dict(fields)
        out.update(tn=tn, time=time, cgrav_old=cgrav_old)
        return out

    def write_bin(self, path: str, exact: bool = False) -> Dict[str, object]:
        self.checkpoint_begin(exact=exact)
        return self.checkpoint_finish(path)

    @classmethod
    def restart(cls, cfg: dict, path: str, precision: int = 0) -> "Simulation":
        """Resume from a dump as restart.f90 does: read it (readbin.f90),
        rebuild U from the primitives (conserve.f90), continue the clock.  If
        the dump has the conserved planes beside it (<path>.u.npy, written
        by an exact checkpoint) they are used instead, and the run resumes
        bit for bit."""
        import os

        f = binio.readbin(path, cfg["n"], bool(cfg["mag_on"]), cfg["gravswitch"], cfg.get("compswitch", 0))
        st = ic.restart_state(cfg, f)
        if os.path.exists(path + ".u.npy"):
            st["u"] = np.ascontiguousarray(np.load(path + ".u.npy"))
        return cls(cfg, None, grvphi=f.get("grvphi"), grvpsi=f.get("grvpsi"), cgrav_old=float(f.get("cgrav_old", 0.0)),
                   precision=precision, _state=st, _clock=(float(f["time"]), int(f["tn"])))

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

    def evo(self) -> Dict[str, float]:
        """One line of evo_output (output.f90:147-275): tn, time and the
        totals the reference writes for this set-up (gravity entries with
        self-gravity, Ebtot with fields, Jtot on curvilinear grids of two or
        more dimensions), doubled with equatorial symmetry."""
        tot = self.ctx.evo()
        c = self.cfg
        keys = ["Mtot", "Etot", "Eitot", "Ektot"]
        if c["gravswitch"] >= 1:
            keys += ["Egtot", "Mbound", "Ebound", "Jbound"]
        if c["mag_on"]:
            keys.append("Ebtot")
        if c["dim"] >= 2 and c.get("crdnt", 0) >= 1:
            keys.append("Jtot")
        f = 2.0 if c.get("eq_sym", False) else 1.0
        out = {"tn": self.tn, "time": self.time}
        out.update({k: f * tot[k] for k in keys})
        return out

    def state(self, gravity: bool = False) -> Dict[str, np.ndarray]:
        out = self.ctx.download(gravity=gravity)
        if self.nspc:
            out["spc"] = self.ctx.download_scalars()
        return out

    def close(self):
        self.ctx.close()
