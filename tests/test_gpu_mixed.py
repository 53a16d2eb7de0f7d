"""The mixed-precision stage (FP32 Riemann solver; FP64 reconstruction,
pressure recovery and compensated accumulation).

It is not bit-compatible, so it is checked by its error against the FP64
form started from the same state, and by exact conservation properties.
The one-step tolerances below are the stated bounds of this form: L1 of
density and total energy <= 1e-6, and for every conserved variable
sum|dq| <= 1e-5 * max(sum|q|, 0.1 * sum|rho|) (fields that are zero or
small are measured against the density scale); the scheme's slope-zeroing test is a
discontinuous switch, so errors over many steps are bounded by the
scheme's own sensitivity (a 1e-14 perturbation of the initial state grows
to ~5e-3 L1 by t=0.5 in 2-D Orszag-Tang, for FP64 too)."""
import numpy as np
import pytest

from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu
PRIM = ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")


def one_step_l1(cfg, prims, warm=3):
    a = Simulation(cfg, prims, precision=0)
    for _ in range(warm):
        a.step()
    st = a.state()
    b = Simulation(cfg, prims, precision=1)
    for s in (a, b):
        s.ctx.upload(u=st["u"], prim=[st[k] for k in PRIM])
        s.time, s.tn = 0.01, 1
    a.step()
    b.step()
    sa, sb = a.state(), b.state()
    a.close()
    b.close()
    nv = sa["u"].shape[0]
    rho = np.sum(np.abs(sa["u"][0]))
    return [float(np.sum(np.abs(sb["u"][q] - sa["u"][q])) / max(np.sum(np.abs(sa["u"][q])), 0.1 * rho))
            for q in range(nv)]


@pytest.mark.parametrize("make", [lambda: cases.ot3d(32), lambda: cases.kh2d(64), lambda: cases.blast3d(16, bc=2),
                                  lambda: cases.golden_case("briowushock_x")])
def test_mixed_one_step_error(make):
    cfg, prims = make()
    l1 = one_step_l1(cfg, prims)
    assert l1[0] <= 1e-6 and l1[4] <= 1e-6, l1  # density, total energy
    assert max(l1) <= 1e-5, l1


def test_mixed_conserves_mass_and_energy_in_a_periodic_box():
    cfg, prims = cases.ot3d(24)
    s = Simulation(cfg, prims, precision=1)
    u0 = s.state()["u"]
    for _ in range(10):
        s.step()
    u1 = s.state()["u"]
    s.close()
    for q in (0, 4):  # mass and total energy: fluxes telescope, sources vanish
        assert abs(u1[q].sum() - u0[q].sum()) <= 1e-12 * abs(u0[q].sum())
