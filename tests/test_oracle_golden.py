"""The CPU oracle reproduces HORMONE's own golden test dumps.

Each case runs the reference's test set-up (``simtype='<name> test'``,
src/main/setup.f90:44-56; flat variants as the CI's flux_limiter='flat'
switch) through the oracle and compares the final state with the committed
fixture of ``tests/<name>.bin`` using the norms of src/main/tests.f90.  The
restatement is expected to be bit-identical, which is stronger than the
reference's own pass criterion (largest L2 norm < test_tol).
"""
import os

import numpy as np
import pytest

from hormone_b200 import config, grid as G, ic
from oracle.oracle import Oracle
import cases
import norms

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [f"{k}_{d}" for k in ("sodshock", "briowushock") for d in "xyz"] + \
        [f"orszagtang_{p}" for p in ("xy", "yz", "xz")] + ["KHinstability", "sedov_default"]
CASES = CASES + [c + "_flat" for c in CASES]



def run_case(name):
    flat = name.endswith("_flat")
    st = name[:-5] if flat else name
    cfg = config.resolve(st + " test", overrides={"flux_limiter": "flat"} if flat else None)
    grid = G.make_grid(cfg)
    o = Oracle(cfg)
    for a in range(3):
        ax = o.axis(a)
        for k in G.AXIS_KEYS:
            assert np.array_equal(ax[k], grid[a][k]), (a, k)
    if cfg["crdnt"] == 2:  # the host's metric factors are the oracle's restatement
        m = o.metric()
        for name, a, key in (("detg1", 0, "detg"), ("idetg1", 0, "idetg"), ("sx1", 0, "sx"),
                             ("sini", 1, "sini"), ("cosi", 1, "cosi"), ("scot", 1, "scot")):
            assert np.array_equal(m[name], grid[a][key]), name
    o.set_prims(ic.make(cfg, grid))
    o.start()
    assert o.run()
    return cfg, o


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name):
    gold = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    cfg, o = run_case(name)
    sc = o.scalars()
    assert sc["tn"] == int(gold["tn"])
    assert sc["time"] == float(gold["time"])
    sim = {k: o.get(k) for k in ("d", "e", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}
    for n in range(cfg["nspc"]):
        sim[f"spc{n}"] = o.get(f"spc{n}")
    res = norms.compare(sim, gold, cfg, dvol=cases.cell_volumes(cfg, G.make_grid(cfg)))
    worst = max(r["L2"] for r in res.values())
    assert worst < cfg["test_tol"], res  # the reference's own criterion (tests.f90:170)
    for lab, r in res.items():
        assert r["identical"], (lab, r)  # bit-identical restatement


def test_norms_detect_a_planted_error():
    """A one-ulp-scale perturbation planted in the oracle output is seen."""
    gold = dict(np.load(os.path.join(HERE, "golden", "sodshock_x.npz")))
    cfg = config.resolve("sodshock_x test")
    sim = {k: gold[k].copy() for k in ("d", "e", "v1", "v2", "v3")}
    sim["d"][0, 0, 250] *= 1.0 + 1e-12
    res = norms.compare(sim, gold, cfg)
    assert not res["d"]["identical"]
    assert res["d"]["L2"] > cfg["test_tol"]
