"""Batches of independent simulations on one GPU (hmn_batch_* of the C ABI).

``Batch`` admits simulations into one device memory pool (admission by
footprint), advances all of them with one persistent launch per phase and
tile kind (each on its own clock), and hands back results.  The result of
every simulation is bit-identical to running it alone through ``Simulation``.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional

import numpy as np

from . import capi, grid as gridmod, ic

_P, _I, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double


def _bind(L):
    if getattr(L, "_hmn_batch_bound", False):
        return L
    L.hmn_batch_footprint.argtypes = [ctypes.POINTER(capi.HmnGrid), ctypes.POINTER(capi.HmnParams)]
    L.hmn_batch_footprint.restype = ctypes.c_size_t
    L.hmn_batch_create.argtypes = [ctypes.c_size_t, _I, _I, _I, ctypes.POINTER(_P)]
    L.hmn_batch_add.argtypes = [_P, ctypes.POINTER(capi.HmnGrid), ctypes.POINTER(capi.HmnParams), capi._DP,
                                capi._DPP, _D, _D, ctypes.POINTER(_I)]
    L.hmn_batch_remove.argtypes = [_P, _I]
    L.hmn_batch_step.argtypes = [_P, _I]
    L.hmn_batch_set_held.argtypes = [_P, ctypes.POINTER(_I)]
    L.hmn_batch_poll.argtypes = [_P, capi._DP, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]
    L.hmn_batch_download.argtypes = [_P, _I, capi._DP, capi._DPP]
    L.hmn_batch_set_schedule.argtypes = [_P, _I, _I, _I]
    L.hmn_batch_set_sweep.argtypes = [_P, _I, _I]
    L.hmn_batch_launch_count.argtypes = [_P]
    L.hmn_batch_launch_count.restype = ctypes.c_longlong
    L.hmn_batch_sync.argtypes = [_P]
    L.hmn_batch_stream.argtypes = [_P]
    L.hmn_batch_stream.restype = _P
    L.hmn_batch_destroy.argtypes = [_P]
    for n in ("hmn_batch_create", "hmn_batch_add", "hmn_batch_remove", "hmn_batch_step", "hmn_batch_poll",
              "hmn_batch_download", "hmn_batch_set_schedule", "hmn_batch_set_sweep", "hmn_batch_sync",
              "hmn_batch_destroy", "hmn_batch_set_held"):
        getattr(L, n).restype = _I
    L._hmn_batch_bound = True
    return L


def footprint(cfg: dict, grid=None) -> int:
    """Device bytes the simulation occupies in a batch pool."""
    L = _bind(capi.lib())
    grid = grid if grid is not None else gridmod.make_grid(cfg)
    gs, keep = capi.grid_struct(cfg, grid)
    ps = capi.params_struct(cfg)
    return int(L.hmn_batch_footprint(ctypes.byref(gs), ctypes.byref(ps)))


class Batch:
    def __init__(self, pool_bytes: int, max_sims: int = 1024, precision: int = 0, rktype: int = 3):
        L = _bind(capi.lib())
        h = _P()
        rc = L.hmn_batch_create(int(pool_bytes), int(max_sims), int(precision), int(rktype), ctypes.byref(h))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_create")
        self.h = h
        self.max_sims = max_sims
        self.pool_bytes = pool_bytes
        self.meta: Dict[int, dict] = {}

    def close(self):
        if getattr(self, "h", None):
            capi.lib().hmn_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, cfg: dict, prims: Optional[Dict[str, np.ndarray]] = None, grid=None, time: float = 0.0,
            t_end: Optional[float] = None) -> Optional[int]:
        """Admit a simulation; returns its slot, or None if it does not fit
        (pool memory or slots exhausted)."""
        L = capi.lib()
        if int(cfg.get("crdnt", 0)) != 0:
            raise ValueError("batches hold Cartesian grids; a curvilinear grid runs as its own Simulation")
        grid = grid if grid is not None else gridmod.make_grid(cfg)
        if prims is None:
            prims = ic.make(cfg, grid)
        st = ic.to_state(cfg, prims)
        gs, keep = capi.grid_struct(cfg, grid)
        ps = capi.params_struct(cfg)
        u = np.ascontiguousarray(st["u"])
        prim = np.ascontiguousarray(st["prim"])
        pp = (capi._DP * 9)()
        for q in range(9):
            pp[q] = capi._dp(prim[q])
        sim = _I()
        rc = L.hmn_batch_add(self.h, ctypes.byref(gs), ctypes.byref(ps), capi._dp(u), pp, float(time),
                             float(cfg["t_end"] if t_end is None else t_end), ctypes.byref(sim))
        if rc == capi.HMN_ENOMEM:
            return None
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_add")
        self.meta[sim.value] = {"cfg": cfg, "shape": (cfg["n"][2], cfg["n"][1], cfg["n"][0]), "nvar": cfg["nvar"]}
        return sim.value

    def capacity(self, cfg: dict) -> bool:
        """Whether a simulation of this configuration could ever fit the pool."""
        return footprint(cfg) <= self.pool_bytes

    def remove(self, sim: int):
        rc = capi.lib().hmn_batch_remove(self.h, int(sim))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_remove")
        self.meta.pop(sim, None)

    def step(self, nsteps: int = 1):
        rc = capi.lib().hmn_batch_step(self.h, int(nsteps))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_step")

    def set_held(self, slots):
        """Leave the simulations in `slots` out of the following steps (and
        release every other one)."""
        held = np.zeros(self.max_sims, dtype=np.int32)
        for s in slots:
            held[int(s)] = 1
        rc = capi.lib().hmn_batch_set_held(self.h, held.ctypes.data_as(ctypes.POINTER(_I)))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_set_held")

    def poll(self):
        n = self.max_sims
        t = np.zeros(n)
        tn, done, err = (np.zeros(n, dtype=np.int32) for _ in range(3))
        rc = capi.lib().hmn_batch_poll(self.h, capi._dp(t), tn.ctypes.data_as(ctypes.POINTER(_I)),
                                       done.ctypes.data_as(ctypes.POINTER(_I)), err.ctypes.data_as(ctypes.POINTER(_I)))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_poll")
        return t, tn, done, err

    def download(self, sim: int) -> Dict[str, np.ndarray]:
        m = self.meta[sim]
        U = np.empty((m["nvar"],) + m["shape"])
        P = np.empty((9,) + m["shape"])
        pp = (capi._DP * 9)()
        for q in range(9):
            pp[q] = capi._dp(P[q])
        rc = capi.lib().hmn_batch_download(self.h, int(sim), capi._dp(U), pp)
        if rc < 0 and rc != capi.HMN_ENEG_EINT:
            raise capi.HmnError(rc, "hmn_batch_download")
        out = {"u": U, "error": rc}
        for q, k in enumerate(("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")):
            out[k] = P[q]
        return out

    def set_schedule(self, kind: int, tile_id: int, blocks_per_sm: int = 0):
        """kind 0 3-D / 1 2-D x-y / 2 1-D x; tile_id per include/hormone_gpu.h."""
        rc = capi.lib().hmn_batch_set_schedule(self.h, int(kind), int(tile_id), int(blocks_per_sm))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_set_schedule")

    def set_sweep(self, kind: int, sweep: int):
        """Work-list order and CTA split of kind's stage launches: 0 static
        (slot order), 1 interleaved across simulations, 2 dynamic (largest
        simulations first, CTAs take items from a shared counter)."""
        rc = capi.lib().hmn_batch_set_sweep(self.h, int(kind), int(sweep))
        if rc != 0:
            raise capi.HmnError(rc, "hmn_batch_set_sweep")

    def sync(self):
        capi.lib().hmn_batch_sync(self.h)

    def launches(self) -> int:
        return int(capi.lib().hmn_batch_launch_count(self.h))

    def stream_ptr(self) -> int:
        return int(capi.lib().hmn_batch_stream(self.h) or 0)

    def run_all(self, chunk: int = 16, max_steps: int = 10 ** 7) -> int:
        """Step until every admitted simulation has reached its end time;
        returns the number of batch steps issued."""
        steps = 0
        while steps < max_steps:
            self.step(chunk)
            steps += chunk
            t, tn, done, err = self.poll()
            live = [s for s in self.meta if not done[s]]
            if any(err[s] for s in self.meta):
                bad = [s for s in self.meta if err[s]]
                raise capi.HmnError(int(err[bad[0]]), "batch step", None)
            if not live:
                break
        return steps
