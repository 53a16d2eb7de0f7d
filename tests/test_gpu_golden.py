"""The GPU path run to completion reproduces HORMONE's golden dumps.

Same comparison as tests.f90:46-182 (and the oracle test), through the C ABI
step loop; the result is expected to be bit-identical to the reference's
committed output."""
import os

import numpy as np
import pytest

from hormone_b200 import grid as G
from hormone_b200.sim import Simulation

import cases
import norms

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = [f"{k}_{d}" for k in ("sodshock", "briowushock") for d in "xyz"] + \
        [f"orszagtang_{p}" for p in ("xy", "yz", "xz")] + ["KHinstability", "sedov_default"]
NAMES = NAMES + [n + "_flat" for n in NAMES]


@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_golden(name):
    gold = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    cfg, prims = cases.golden_case(name)
    s = Simulation(cfg, prims)
    assert s.run()
    assert s.tn == int(gold["tn"]) and s.time == float(gold["time"])
    st = s.state()
    s.close()
    for n in range(cfg["nspc"]):
        st[f"spc{n}"] = st["spc"][n]
    res = norms.compare(st, gold, cfg, dvol=cases.cell_volumes(cfg, G.make_grid(cfg)))
    assert max(r["L2"] for r in res.values()) < cfg["test_tol"], res
    for lab, r in res.items():
        assert r["identical"], (lab, r)


def test_device_loop_equals_host_loop():
    """hmn_run (device-resident time, no per-step host sync) gives the same
    state as the per-call drop-in loop."""
    cfg, prims = cases.golden_case("orszagtang_xy")
    a = Simulation(cfg, prims)
    b = Simulation(cfg, prims)
    for _ in range(40):
        a.step()
    b.run_device(max_steps=40)
    assert a.tn == b.tn and a.time == b.time
    sa, sb = a.state(), b.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["briowushock_x", "sedov_default", "orszagtang_xy_flat"])
def test_device_loop_to_end_matches_golden(name):
    """hmn_run to the end time: one plain step, then CUDA-graph replays of
    16 steps whose overshoot past the end does nothing on the device."""
    gold = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    cfg, prims = cases.golden_case(name)
    s = Simulation(cfg, prims)
    assert s.run_device()
    assert s.tn == int(gold["tn"]) and s.time == float(gold["time"])
    st = s.state()
    for k in ("d", "e", "v1", "v2", "v3", "b1", "b2", "b3"):
        if k in gold:
            assert np.array_equal(st[k], gold[k]), k
    s.close()


def test_device_loop_in_pieces_equals_one_call():
    """Calls of hmn_run that stop and restart (odd step counts, so the
    graph is entered on either primitive buffer) give the state of one call."""
    cfg, prims = cases.golden_case("orszagtang_xy")
    a = Simulation(cfg, prims)
    b = Simulation(cfg, prims)
    a.run_device(max_steps=77)
    for n in (33, 1, 19, 24):
        b.run_device(max_steps=n)
    assert a.tn == b.tn == 77 and a.time == b.time
    sa, sb = a.state(), b.state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k]), k
    a.close()
    b.close()
