"""Autotuner for batched steps: tile shape, persistent-grid size and sweep
schedule.

For every grid kind present in a batch (3-D, 2-D x-y, 1-D x) it times each
candidate schedule on a scratch batch holding a sample of the real
simulations, keeps the fastest, and caches it in a JSON file keyed by kind,
precision and size class.  A candidate is

- a tile variant of the kind (8x8x8 or 8x8x4 tiles in 3-D, 16x16 or 32x8 in
  2-D, 256 cells in 1-D),
- a stage-launch grid in CTAs per SM (0: the occupancy limit; above it the
  launch is no longer persistent and CTAs run in waves), and
- a sweep schedule (``hmn_batch_set_sweep``): the work list in slot order
  split statically over the CTAs, interleaved across simulations, or largest
  simulations first taken dynamically from a shared counter.

Schedules never change results (each cell is computed the same way whatever
the tiling, order or split), only speed.
"""
from __future__ import annotations

import json
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

TILE_VARIANTS = {0: (0, 1), 1: (2, 3), 2: (4,)}  # tile ids per kind (include/hormone_gpu.h)
GRID_SIZES = (0, 1, 2, 4)                          # CTAs per SM; 0 = occupancy limit
SWEEPS = (0, 1, 2)                                 # HMN_SWEEP_STATIC, _INTERLEAVED, _DYNAMIC
DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "hormone_b200", "autotune.json")


def grid_kind(cfg) -> int:
    s = [n > 1 for n in cfg["n"]]
    if all(s):
        return 0
    if s[0] and s[1] and not s[2]:
        return 1
    if s[0] and not s[1] and not s[2]:
        return 2
    return -1


def size_class(cells: int) -> int:
    return int(np.log2(max(cells, 1)))


def _load(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _save(path, data):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
    except OSError:
        pass


def time_steps(batch, steps: int) -> float:
    """Milliseconds per batch step, timed with CUDA events on the batch's stream."""
    import torch

    stream = torch.cuda.ExternalStream(batch.stream_ptr())
    batch.step(1)  # builds the graph for the current schedule
    batch.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / steps


def candidates(kind: int) -> List[Tuple[int, int, int]]:
    """Every (tile_id, blocks_per_sm, sweep) the tuner times for ``kind``."""
    return [(t, g, w) for t in TILE_VARIANTS[kind] for g in GRID_SIZES for w in SWEEPS]


def tune(sample: List[Tuple[dict, dict]], precision: int = 0, steps: int = 3, cache: Optional[str] = DEFAULT_CACHE,
         pool_bytes: Optional[int] = None) -> Dict[int, Tuple[int, int, int]]:
    """Best (tile_id, blocks_per_sm, sweep) per grid kind for simulations like
    ``sample`` (a list of (cfg, prims)).  Uses and updates ``cache``."""
    from .batch import Batch, footprint

    by_kind: Dict[int, List[Tuple[dict, dict]]] = {}
    for cfg, prims in sample:
        k = grid_kind(cfg)
        if k >= 0:
            by_kind.setdefault(k, []).append((cfg, prims))
    data = _load(cache) if cache else {}
    best: Dict[int, Tuple[int, int, int]] = {}
    for kind, sims in by_kind.items():
        cells = int(np.mean([np.prod(c["n"]) for c, _ in sims]))
        key = f"k{kind}_p{precision}_s{size_class(cells)}_n{min(len(sims), 64)}"
        if key in data and len(data[key].get("schedule", ())) == 3:
            best[kind] = tuple(data[key]["schedule"])
            continue
        need = sum(footprint(c) for c, _ in sims) + (1 << 24)
        b = Batch(pool_bytes or need, max_sims=len(sims) + 1, precision=precision)
        for cfg, prims in sims:
            b.add(cfg, prims, t_end=1e30)
        results = []
        for tid, g, w in candidates(kind):
            b.set_schedule(kind, tid, g)
            b.set_sweep(kind, w)
            results.append((time_steps(b, steps), tid, g, w))
        b.close()
        results.sort()
        best[kind] = tuple(results[0][1:])
        data[key] = {"schedule": list(best[kind]), "ms_per_step": results[0][0],
                     "candidates": [[r[1], r[2], r[3], r[0]] for r in results]}
    if cache:
        _save(cache, data)
    return best


def apply(batch, schedule: Dict[int, Tuple[int, ...]]):
    """Set each kind's (tile_id, blocks_per_sm[, sweep]) on ``batch``."""
    for kind, sched in schedule.items():
        batch.set_schedule(kind, sched[0], sched[1])
        batch.set_sweep(kind, sched[2] if len(sched) > 2 else 0)
