"""Serving loop: continuous batching of simulation requests on one GPU.

Requests arrive over time (a seeded Poisson stream in the benchmark).  The
server admits each arrived request into the running batch as soon as the
batch's device pool has room for its footprint (first come, first served,
or shortest estimated work first under a cap on the live cells, with
smaller requests allowed to pass a head-of-line request that does not fit),
advances all admitted simulations together a few steps at a time (each
on its own clock), and retires every simulation that reached its end time:
its result is copied back, its pool memory is freed for waiting requests.
Reported: time-to-solution per request (completion minus arrival, wall
clock), its p50/p99, and the aggregate zone-updates/s of the stream.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import config, grid as gridmod, ic

PI = math.acos(-1.0)


@dataclass
class Request:
    rid: int
    cfg: dict
    prims: Dict[str, np.ndarray]
    arrival: float            # seconds after the start of the stream
    cells: int = 0
    kind: str = ""
    result: Optional[dict] = None
    steps: int = 0
    t_admit: float = math.nan
    t_done: float = math.nan
    error: int = 0

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def make_requests(n: int, rate: float, seed: int = 20261203, max_cells: int = 128 ** 3, min_cells: int = 256,
                  sedov_fraction: float = 0.25) -> List[Request]:
    """A seeded request stream: MHD Riemann problems (1-D/2-D/3-D) and Sedov
    blasts, cells log-uniform in [min_cells, max_cells], Poisson arrivals at
    `rate` per second.  Riemann states: rho, p log-U[0.01, 10], v, B U[-1, 1],
    gamma from {5/3, 1.4, 2}; t_end U[0.05, 0.2]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    out = []
    for r in range(n):
        sedov = rng.uniform() < sedov_fraction
        dim = 3 if sedov else int(rng.integers(1, 4))
        cells = math.exp(rng.uniform(math.log(min_cells), math.log(max_cells)))
        edge = {1: 16384, 2: 1024, 3: 128}[dim]
        n_ax = int(min(max(round(cells ** (1.0 / dim)), 8), edge))
        t_end = float(rng.uniform(0.05, 0.2))
        if sedov:
            ov = dict(ie=n_ax, je=n_ax, ke=n_ax, mag_on=False, gamma=1.6666666666666667, flux_limiter="minmod",
                      courant=0.4, t_end=t_end, dt_out=t_end)
            for a in (1, 2, 3):
                for tag in ("is", "os", "iv", "ov"):
                    ov[f"bc{a}{tag}"] = 2
            cfg = config.resolve("sedov_cartesian", overrides=ov)
            prims = ic.sedov(cfg, gridmod.make_grid(cfg), energy=1.0, radius=0.05, rho0=1.0, p0=1e-5)
            kind = "sedov3d"
        else:
            gamma = float(rng.choice([1.6666666666666667, 1.4, 2.0]))
            ns = [n_ax if d < dim else 1 for d in range(3)]
            ov = dict(ie=ns[0], je=ns[1], ke=ns[2], mag_on=True, gamma=gamma, flux_limiter="minmod", courant=0.4,
                      t_end=t_end, dt_out=t_end)
            for a in (1, 2, 3):
                for tag in ("is", "os", "iv", "ov"):
                    ov[f"bc{a}{tag}"] = 3
            cfg = config.resolve("riemann", overrides=ov)
            states = [dict(d=float(np.exp(rng.uniform(math.log(0.01), math.log(10.0)))),
                           p=float(np.exp(rng.uniform(math.log(0.01), math.log(10.0)))),
                           v1=float(rng.uniform(-1, 1)), v2=float(rng.uniform(-1, 1)), v3=float(rng.uniform(-1, 1)),
                           b1=float(rng.uniform(-1, 1)), b2=float(rng.uniform(-1, 1)), b3=float(rng.uniform(-1, 1)))
                      for _ in range(2)]
            states[1]["b1"] = states[0]["b1"]  # the normal field is continuous across the interface
            prims = ic.riemann(cfg, 0, states[0], states[1])
            kind = f"riemann{dim}d"
        out.append(Request(r, cfg, prims, float(arrivals[r]), cells=int(np.prod(cfg["n"])), kind=kind))
    return out


@dataclass
class ServeStats:
    completed: int = 0
    failed: int = 0
    wall_s: float = 0.0
    zone_updates: float = 0.0
    latencies: List[float] = field(default_factory=list)
    max_live: int = 0
    batch_steps: int = 0
    failures: List[tuple] = field(default_factory=list)  # (request id, kind, cells, error code, steps)

    def summary(self) -> dict:
        lat = np.array(self.latencies) if self.latencies else np.zeros(1)
        return {"completed": self.completed, "failed": self.failed, "failures": self.failures[:20],
                "wall_s": self.wall_s,
                "zone_updates_per_s": self.zone_updates / max(self.wall_s, 1e-12),
                "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                "max_concurrent": self.max_live, "batch_steps": self.batch_steps}


def estimated_work(cfg: dict) -> float:
    """Zone-updates a request needs, up to a constant: its cells times its
    steps, which grow with t_end and, through the CFL condition on the
    finest width, with the cells along its longest axis."""
    n = [int(v) for v in cfg["n"]]
    return float(np.prod(n)) * max(n) * float(cfg["t_end"])


def serve(requests: List[Request], batch, chunk: int = 8, clock: Callable[[], float] = time.perf_counter,
          keep_results: bool = True, realtime: bool = True, policy: str = "fifo",
          live_cells: Optional[int] = None, boost: int = 8, short_frac: float = 0.05) -> ServeStats:
    """Run the stream through `batch` (a hormone_b200.batch.Batch or any
    object with add/step/poll/download/remove).  With realtime=False arrival
    times are ignored (every request is available at once).

    policy "fifo" admits arrived requests in arrival order; "sjf" in order of
    estimated work (shortest first, arrival order among equals).  live_cells
    caps the cells of the admitted simulations (a request larger than the
    cap still runs when nothing else does): every batch step advances every
    live simulation, so a small request admitted beside many large ones
    waits for as many of their steps as it needs itself.

    policy "priority" admits in arrival order and, after every `chunk`
    steps of all live simulations, holds the large ones (more cells than
    short_frac of the largest live one) and advances the small ones alone
    for boost x chunk more steps: a small request no longer pays for the
    large ones' cells at every one of its steps.  (Needs a batch with
    set_held.)  Every simulation still takes exactly its own steps, so the
    results do not depend on the policy."""
    if policy not in ("fifo", "sjf", "priority"):
        raise ValueError(f"unknown admission policy {policy!r}")
    stats = ServeStats()
    pending = sorted(requests, key=lambda r: r.arrival)
    waiting: List[Request] = []
    running: Dict[int, Request] = {}
    t0 = clock()
    i = 0
    while i < len(pending) or waiting or running:
        now = clock() - t0
        while i < len(pending) and (not realtime or pending[i].arrival <= now):
            waiting.append(pending[i])
            i += 1
        if policy == "sjf":
            waiting.sort(key=lambda r: estimated_work(r.cfg))  # stable: arrival order among equals
        # admission in policy order, letting smaller requests pass one that does not fit yet
        still = []
        live = sum(r.cells for r in running.values())
        for r in waiting:
            cap = getattr(batch, "capacity", None)
            if cap is not None and cap(r.cfg) is False:  # can never fit: fail it instead of waiting forever
                r.error = -5
                r.t_done = clock() - t0
                stats.failed += 1
                stats.failures.append((r.rid, r.kind, r.cells, r.error, 0))
                continue
            if live_cells is not None and running and live + r.cells > live_cells:
                still.append(r)
                continue
            slot = batch.add(r.cfg, r.prims)
            if slot is None:
                still.append(r)
                continue
            r.t_admit = clock() - t0
            running[slot] = r
            live += r.cells
        waiting = still
        stats.max_live = max(stats.max_live, len(running))
        if not running:
            if i < len(pending) and realtime:
                time.sleep(max(0.0, min(pending[i].arrival - (clock() - t0), 0.01)))
            continue
        batch.step(chunk)
        stats.batch_steps += chunk
        if policy == "priority" and len(running) > 1:
            top = max(r.cells for r in running.values())
            held = [s for s, r in running.items() if r.cells > short_frac * top]
            if len(held) < len(running):
                batch.set_held(held)
                batch.step(boost * chunk)
                batch.set_held([])
                stats.batch_steps += boost * chunk
        _, tn, done, err = batch.poll()
        for slot in [s for s in running if done[s] or err[s]]:
            r = running.pop(slot)
            res = batch.download(slot)
            r.steps = int(tn[slot])
            r.error = int(err[slot])
            r.t_done = clock() - t0
            if keep_results:
                r.result = res
            batch.remove(slot)
            if r.error:
                stats.failed += 1
                stats.failures.append((r.rid, r.kind, r.cells, r.error, r.steps))
            else:
                stats.completed += 1
                stats.latencies.append(r.latency)
                stats.zone_updates += r.cells * r.steps
    stats.wall_s = clock() - t0
    return stats
