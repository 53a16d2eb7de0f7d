"""Serving: requests that arrive while others run are admitted as memory
frees up, and each result is the same alone and in the mix."""
import numpy as np
import pytest

from hormone_b200 import serve
from hormone_b200.batch import Batch, footprint
from hormone_b200.sim import Simulation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("policy", ["fifo", "sjf", "priority"])
def test_continuous_batching_results_equal_alone(policy):
    """Under every admission and stepping policy (with "priority" the large
    simulations are held while the small ones take extra steps)."""
    reqs = serve.make_requests(10, rate=200.0, seed=5, max_cells=24 ** 3, min_cells=64)
    for r in reqs:
        r.cfg = dict(r.cfg)
        r.cfg["t_end"] = min(r.cfg["t_end"], 0.01)
    pool = max(footprint(r.cfg) for r in reqs) * 3  # forces queueing: at most ~3 at once
    b = Batch(pool, max_sims=16)
    stats = serve.serve(reqs, b, chunk=2, policy=policy, live_cells=20000 if policy == "sjf" else None,
                        short_frac=0.2)
    b.close()
    assert stats.completed + stats.failed == len(reqs)
    assert stats.max_live >= 2  # work overlapped
    for r in reqs:
        if r.error:
            continue
        s = Simulation(r.cfg, r.prims)
        s.run_device()
        st = s.state()
        s.close()
        assert s.tn == r.steps
        for k in ("u", "d", "v1", "e", "b1", "phi"):
            assert np.array_equal(st[k], r.result[k]), (r.rid, k)
    summ = stats.summary()
    assert summ["p99_s"] >= summ["p50_s"] >= 0.0


def test_held_simulation_keeps_its_clock_and_state():
    """hmn_batch_set_held: a held simulation is left out of the steps (clock
    and state unchanged), and once released it ends with the same bits as
    when run alone."""
    reqs = serve.make_requests(2, rate=1e9, seed=8, max_cells=16 ** 3, min_cells=512)
    for r in reqs:
        r.cfg = dict(r.cfg)
        r.cfg["t_end"] = min(r.cfg["t_end"], 0.01)
    b = Batch(sum(footprint(r.cfg) for r in reqs) * 2, max_sims=4)
    a = b.add(reqs[0].cfg, reqs[0].prims)
    c = b.add(reqs[1].cfg, reqs[1].prims)
    b.step(3)
    t0, tn0, _, _ = b.poll()
    before = b.download(c)
    b.set_held([c])
    b.step(5)
    t1, tn1, _, _ = b.poll()
    assert tn1[c] == tn0[c] and t1[c] == t0[c] and tn1[a] > tn0[a]
    after = b.download(c)
    for k in before:
        assert np.array_equal(before[k], after[k]), k
    b.set_held([])
    for _ in range(10000):
        _, tn, done, err = b.poll()
        if done[a] and done[c]:
            break
        b.step(8)
    for slot, r in ((a, reqs[0]), (c, reqs[1])):
        got = b.download(slot)
        s = Simulation(r.cfg, r.prims)
        s.run_device()
        st = s.state()
        s.close()
        assert s.tn == tn[slot] and not err[slot]
        for k in ("u", "d", "v1", "e", "b1", "phi"):
            assert np.array_equal(st[k], got[k]), (slot, k)
    b.close()
