"""Serving: requests that arrive while others run are admitted as memory
frees up, and each result is the same alone and in the mix."""
import numpy as np
import pytest

from hormone_b200 import serve
from hormone_b200.batch import Batch, footprint
from hormone_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def test_continuous_batching_results_equal_alone():
    reqs = serve.make_requests(10, rate=200.0, seed=5, max_cells=24 ** 3, min_cells=64)
    for r in reqs:
        r.cfg = dict(r.cfg)
        r.cfg["t_end"] = min(r.cfg["t_end"], 0.01)
    pool = max(footprint(r.cfg) for r in reqs) * 3  # forces queueing: at most ~3 at once
    b = Batch(pool, max_sims=16)
    stats = serve.serve(reqs, b, chunk=2)
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
