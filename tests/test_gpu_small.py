"""Small grids run whole steps in one persistent launch (hmn_small.cu): the
state after N steps is bitwise that of the per-phase launches (HMN_SMALL=0:
CFL, dt, rktype stages and advance as separate kernels in CUDA graphs), on
1-D, 2-D and 3-D grids, hydro and MHD with GLM, Cartesian and spherical,
rk2 and rk3, and when the steps are split over several calls (the pending
phidamp factor and the primitive-buffer parity carry across)."""
import numpy as np
import pytest

from hormone_b200 import config, grid as G, ic
from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def brio_wu_1024():
    cfg = config.resolve("briowushock_x test", overrides=dict(ie=1024, t_end=100.0, dt_out=100.0, courant=0.4,
                                                              flux_limiter="minmod"))
    return cfg, ic.make(cfg, G.make_grid(cfg))


CASES = {
    "brio-wu-1024": brio_wu_1024,
    "sedov-spherical": lambda: cases.golden_case("sedov_default"),
    "orszag-tang-2d-glm": lambda: cases.golden_case("orszagtang_xy"),
    "kh-2d-rk2": lambda: _rk2(cases.kh2d(48)),
    "blast-3d-hydro": lambda: cases.blast3d(16, bc=2),
    "orszag-tang-3d-glm": lambda: cases.ot3d(16),
}


def _rk2(case):
    cfg, prims = case
    cfg = dict(cfg)
    cfg["rktype"] = 2
    return cfg, prims


def run(cfg, prims, pieces, small, monkeypatch):
    monkeypatch.setenv("HMN_SMALL", "1" if small else "0")
    s = Simulation(cfg, prims)
    for n in pieces:
        s.run_device(max_steps=n)
    st = s.state()
    st["tn"], st["time"] = s.tn, s.time
    s.close()
    return st


@pytest.mark.parametrize("name", sorted(CASES))
def test_persistent_small_grid_loop_equals_per_phase_launches(name, monkeypatch):
    cfg, prims = CASES[name]()
    assert int(np.prod(cfg["n"])) <= 65536
    ref = run(cfg, prims, [60], False, monkeypatch)
    for pieces in ([60], [7, 1, 33, 19]):
        got = run(cfg, prims, pieces, True, monkeypatch)
        assert got["tn"] == ref["tn"] == 60 and got["time"] == ref["time"], (pieces, got["tn"], ref["tn"])
        for k in ref:
            if isinstance(ref[k], np.ndarray):
                assert np.array_equal(got[k], ref[k]), (name, pieces, k)


def test_persistent_loop_stops_at_the_end_time(monkeypatch):
    """A run to t_end in one call: the device clock ends the loop, and the
    state equals the per-phase launches' run to the same end."""
    cfg, prims = cases.golden_case("briowushock_x")
    a = run(cfg, prims, [10 ** 6], False, monkeypatch)
    b = run(cfg, prims, [10 ** 6], True, monkeypatch)
    assert a["tn"] == b["tn"] and a["time"] == b["time"]
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
