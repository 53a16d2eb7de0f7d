"""Batched simulations (hmn_batch_*): every simulation in a batch gives the
same bits as the same simulation run alone, whatever else is in the batch,
whatever tile and persistent-grid schedule, and admission follows the pool's
free memory."""
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


def test_schedule_does_not_change_results():
    sims = mix()[:4]
    outs = []
    for sched in ({0: (0, 0), 1: (2, 0)}, {0: (1, 1), 1: (3, 2)}):
        b = Batch(sum(footprint(c) for c, _ in sims) + (1 << 20), max_sims=8)
        slots = [b.add(c, p) for c, p in sims]
        autotune.apply(b, sched)
        b.step(5)
        outs.append([b.download(s)["u"] for s in slots])
        b.close()
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


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


def test_autotuner_picks_a_valid_schedule(tmp_path):
    sims = mix()[:3]
    best = autotune.tune(sims, steps=2, cache=str(tmp_path / "tune.json"))
    assert set(best) == {1}
    tid, g = best[1]
    assert tid in autotune.TILE_VARIANTS[1] and g in autotune.GRID_SIZES
    again = autotune.tune(sims, steps=2, cache=str(tmp_path / "tune.json"))  # served from the cache
    assert again == best
