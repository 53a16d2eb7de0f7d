"""Host logic of the batch autotuner (no GPU): the search space is tiles x
grid sizes x sweep schedules, the fastest timed candidate wins, the cache
serves it back, and a cached entry from the older two-field schedule is
tuned again."""
import json

import pytest

from hormone_b200 import autotune, batch as batchmod

import cases


class FakeBatch:
    """Records the schedule it is given; `cost` maps a schedule to ms."""

    made = []

    def __init__(self, pool_bytes, max_sims=1, precision=0):
        self.sched, self.sweep, self.added, self.closed = {}, {}, 0, False
        FakeBatch.made.append(self)

    def add(self, cfg, prims, t_end=None):
        self.added += 1
        return self.added - 1

    def set_schedule(self, kind, tid, g):
        assert tid in autotune.TILE_VARIANTS[kind] and g in autotune.GRID_SIZES
        self.sched[kind] = (tid, g)

    def set_sweep(self, kind, w):
        assert w in autotune.SWEEPS
        self.sweep[kind] = w

    def close(self):
        self.closed = True


def cost(b):
    # a made-up landscape with its minimum at 32x8 tiles, 2 CTAs/SM, dynamic sweep
    (tid, g), w = b.sched[1], b.sweep[1]
    return 1.0 + 0.5 * (tid != 3) + 0.25 * abs(g - 2) + 0.125 * (w != 2)


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.made = []
    monkeypatch.setattr(batchmod, "Batch", FakeBatch)
    monkeypatch.setattr(batchmod, "footprint", lambda cfg: 1 << 20)
    monkeypatch.setattr(autotune, "time_steps", lambda b, steps: cost(b))
    return FakeBatch


def test_search_space_is_tiles_by_grids_by_sweeps():
    for kind, tiles in autotune.TILE_VARIANTS.items():
        c = autotune.candidates(kind)
        assert len(c) == len(set(c)) == len(tiles) * len(autotune.GRID_SIZES) * len(autotune.SWEEPS)
        assert {x[0] for x in c} == set(tiles)
        assert {x[1] for x in c} == set(autotune.GRID_SIZES)
        assert {x[2] for x in c} == set(autotune.SWEEPS)


def test_tune_keeps_the_fastest_candidate_and_caches_it(fake, tmp_path):
    sims = [cases.kh2d(16), cases.kh2d(24)]
    path = tmp_path / "t.json"
    best = autotune.tune(sims, cache=str(path))
    assert best == {1: (3, 2, 2)}
    assert len(fake.made) == 1 and fake.made[0].added == 2 and fake.made[0].closed
    entry = next(iter(json.loads(path.read_text()).values()))
    assert entry["schedule"] == [3, 2, 2] and entry["ms_per_step"] == 1.0
    assert len(entry["candidates"]) == len(autotune.candidates(1))
    # a second call is served from the cache: no scratch batch
    assert autotune.tune(sims, cache=str(path)) == best and len(fake.made) == 1


def test_two_field_cache_entries_are_tuned_again(fake, tmp_path):
    sims = [cases.kh2d(16)]
    path = tmp_path / "t.json"
    autotune.tune(sims, cache=str(path))
    data = json.loads(path.read_text())
    key = next(iter(data))
    data[key] = {"schedule": [2, 0], "ms_per_step": 1.0, "candidates": []}
    path.write_text(json.dumps(data))
    assert autotune.tune(sims, cache=str(path)) == {1: (3, 2, 2)}
    assert len(fake.made) == 2


def test_apply_sets_tile_grid_and_sweep():
    b = FakeBatch(0)
    autotune.apply(b, {1: (3, 4, 1), 0: (0, 0)})  # a two-field schedule means the static sweep
    assert b.sched == {1: (3, 4), 0: (0, 0)} and b.sweep == {1: 1, 0: 0}
