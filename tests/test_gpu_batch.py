"""Batched simulations (hmn_batch_*): every simulation in a batch gives the
same bits as the same simulation run alone, whatever else is in the batch,
whatever tile, persistent-grid size and sweep schedule, and admission follows
the pool's free memory."""
import numpy as np
import pytest

from hormone_b200 import autotune, config, grid as G, ic
from hormone_b200.batch import Batch, footprint
from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def kh_box(n, ratio, bx, seed=0):
    cfg, prims = cases.kh2d(n, ratio=ratio, bx=bx)
    cfg = dict(cfg)
    cfg["t_end"] = 0.05
    return cfg, prims


def mix():
    sims = [kh_box(24, 1.5, 0.02), kh_box(40, 3.0, 0.08), kh_box(17, 2.0, 0.0)]
    c, p = cases.ot3d(12)
    c = dict(c); c["t_end"] = 0.02
    sims.append((c, p))
    c, p = cases.golden_case("briowushock_x")
    c = dict(c); c["t_end"] = 0.02
    sims.append((c, p))
    c, p = cases.blast3d(10, bc=3, mag=False)
    c = dict(c); c["t_end"] = 0.01
    sims.append((c, p))
    for code in (4, 5):  # linear extrapolation, and with outflow only, on every face
        c, p = cases.blast3d(9, bc=code, mag=True)
        c = dict(c); c["t_end"] = 0.01
        sims.append((c, p))
    return sims


def alone(cfg, prims, precision=0):
    s = Simulation(cfg, prims, precision=precision)
    s.run_device()
    st = s.state()
    st["tn"], st["time"] = s.tn, s.time
    s.close()
    return st


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_matches_each_simulation_alone(precision):
    sims = mix()
    ref = [alone(c, p, precision) for c, p in sims]
    b = Batch(sum(footprint(c) for c, _ in sims) + (1 << 20), max_sims=16, precision=precision)
    slots = [b.add(c, p) for c, p in sims]
    assert None not in slots
    b.run_all(chunk=4)
    t, tn, done, err = b.poll()
    for s, r in zip(slots, ref):
        assert done[s] and err[s] == 0
        assert tn[s] == r["tn"] and t[s] == r["time"]
        got = b.download(s)
        for k in ("u", "d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi"):
            assert np.array_equal(got[k], r[k]), (s, k)
    b.close()


SCHEDULES = (  # kind -> (tile_id, blocks_per_sm, sweep): every tile, grid size and sweep at least once
    {0: (0, 0, 0), 1: (2, 0, 0), 2: (4, 0, 0)},
    {0: (1, 1, 1), 1: (3, 2, 1), 2: (4, 4, 1)},
    {0: (0, 4, 2), 1: (2, 1, 2), 2: (4, 2, 2)},
    {0: (1, 2, 2), 1: (3, 4, 2), 2: (4, 1, 0)},
)


@pytest.mark.parametrize("precision", [0, 1])
def test_schedule_does_not_change_results(precision):
    """Tile shape, grid size and sweep (static, interleaved, dynamic) give
    the same bits, also when the schedule changes between steps (the work
    list and graph are rebuilt) and over many replays of one graph (the
    dynamic queue resets itself after every launch)."""
    sims = mix()[:5]  # 2-D, 3-D and 1-D kinds
    outs = []
    for i, sched in enumerate(SCHEDULES):
        b = Batch(sum(footprint(c) for c, _ in sims) + (1 << 20), max_sims=8, precision=precision)
        slots = [b.add(c, p) for c, p in sims]
        autotune.apply(b, sched)
        b.step(2)
        autotune.apply(b, SCHEDULES[(i + 1) % len(SCHEDULES)])
        b.step(6)
        t, tn, done, err = b.poll()
        outs.append([(tn[s], t[s], b.download(s)) for s in slots])
        b.close()
    for other in outs[1:]:
        for (tn0, t0, x), (tn1, t1, y) in zip(outs[0], other):
            assert tn0 == tn1 and t0 == t1
            for k in ("u", "d", "v1", "v2", "v3", "e", "b1", "b2", "b3"):
                assert np.array_equal(x[k], y[k]), k


def test_admission_by_footprint_and_slot_reuse():
    c1, p1 = kh_box(32, 2.0, 0.05)
    fp = footprint(c1)
    b = Batch(fp + fp // 2, max_sims=4)
    s1 = b.add(c1, p1)
    assert s1 is not None
    assert b.add(c1, p1) is None  # no room for a second one
    b.step(2)
    b.remove(s1)
    s2 = b.add(c1, p1)  # freed memory is reused
    assert s2 is not None
    b.close()


def test_autotuner_times_every_candidate_and_keeps_the_fastest(tmp_path):
    import json

    sims = mix()[:3]
    path = tmp_path / "tune.json"
    best = autotune.tune(sims, steps=2, cache=str(path))
    assert set(best) == {1}
    entry = next(iter(json.loads(path.read_text()).values()))
    timed = {tuple(c[:3]): c[3] for c in entry["candidates"]}
    assert set(timed) == set(autotune.candidates(1))  # tiles x grid sizes x sweeps
    assert all(ms > 0 for ms in timed.values())
    assert timed[best[1]] == min(timed.values()) == entry["ms_per_step"]
    again = autotune.tune(sims, steps=2, cache=str(path))  # served from the cache
    assert again == best
    # the chosen schedule gives each simulation's own bits
    b = Batch(sum(footprint(c) for c, _ in sims) + (1 << 20), max_sims=4)
    slots = [b.add(c, p) for c, p in sims]
    autotune.apply(b, best)
    b.run_all(chunk=4)
    for s, (c, p) in zip(slots, sims):
        ref = alone(c, p)
        assert np.array_equal(b.download(s)["u"], ref["u"])
    b.close()
