"""How far the FP64 scheme moves when its initial state moves a little.

HORMONE zeroes all slopes of a cell when a face's internal energy falls
outside its neighbours' range (src/main/interpolation.f90:147-163).  At a
contact or any region of nearly uniform pressure that comparison is decided
by the last bits of the face energy, so a tiny change of the state can flip
it.  A flip moves the solution by far more than the change that caused it.
This bounds what any reordering or reduced-precision form of the flux can
match over a whole run: the mixed-precision form is judged per step, and
whole runs against this sensitivity (tests/test_gpu_mixed.py).

Brio-Wu, 1024 cells, minmod, CFL 0.4, to t=0.1 (1944 steps); density and
pressure multiplied by 1 + eps*U[-1,1].  Measured with the oracle over six
seeds: eps = 1e-11 and 1e-10 stay linear (L1(rho) = 4.5-5.4e-12 and
4.5-5.4e-11); at eps = 1e-9 four seeds of six end 3.3e-5 away, at 1e-8 five
of six end 3.3-5.5e-5 away.
"""
import numpy as np

from hormone_b200 import config, grid as G, ic
from oracle.oracle import Oracle


def _run(cfg, prims):
    o = Oracle(cfg)
    o.set_prims(prims)
    o.start()
    while not o.step():
        pass
    return o.get("d")


def test_brio_wu_sensitivity_to_initial_perturbations():
    cfg = config.resolve("briowushock_x test", overrides=dict(ie=1024, t_end=100.0, dt_out=100.0, courant=0.4,
                                                              flux_limiter="minmod"))
    p = ic.make(cfg, G.make_grid(cfg))
    d0 = _run(cfg, p)

    def moved(eps, seed):
        rng = np.random.default_rng(seed)
        q = {k: v.copy() for k, v in p.items()}
        q["p"] = q["p"] * (1 + eps * rng.uniform(-1, 1, size=q["p"].shape))
        q["d"] = q["d"] * (1 + eps * rng.uniform(-1, 1, size=q["d"].shape))
        d1 = _run(cfg, q)
        return float(np.sum(np.abs(d1 - d0)) / np.sum(np.abs(d0)))

    assert moved(1e-11, 0) < 1e-10                       # small changes stay small ...
    assert max(moved(1e-9, s) for s in (0, 1)) > 1e-5   # ... until one flips a slope-zeroing decision


def test_random_riemann_state_flips_within_one_step():
    """On a 3-D MHD state with random left/right Riemann data modulated in y
    and z, the slope-zeroing comparisons sit at their knife edge in many
    cells: one FP64 step from a state whose density and pressure moved by
    1e-12 ends 5e-5 away in L1(rho), while a smooth Orszag-Tang state moves
    linearly.  A per-step bound of 1e-6 for any reordered or reduced-precision
    flux therefore holds on smooth states only."""
    import sys
    import os

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import cases

    def one_step_gap(cfg, prims, eps):
        o = Oracle(cfg)
        o.set_prims(prims)
        o.start()
        for _ in range(3):
            o.step()
        st = {k: o.get(k) for k in ("d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi")}
        rng = np.random.default_rng(1)
        moved = {k: (v * (1 + eps * rng.uniform(-1, 1, v.shape)) if k in ("d", "p") else v) for k, v in st.items()}
        out = []
        for s in (st, moved):
            a = Oracle(cfg)
            a.set_prims(s)
            a.start()
            a.step()
            out.append(a.get("d"))
        return float(np.sum(np.abs(out[1] - out[0])) / np.sum(np.abs(out[0])))

    cfg, prims = cases.riemann3d(n=(24, 16, 12), bc=(3, 3, 3))
    assert one_step_gap(cfg, prims, 1e-12) > 1e-5
    cfg, prims = cases.ot3d(25)
    assert one_step_gap(cfg, prims, 1e-12) < 1e-11
