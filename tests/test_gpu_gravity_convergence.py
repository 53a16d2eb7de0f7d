"""Hyperbolic self-gravity against the analytic potential, independently of
the oracle.

The reference solves hyperbolic gravity only on curvilinear grids and ships
no golden dump of it that this path can reproduce, so the GPU-vs-oracle
parity of the potential (test_gpu_parity.py) rests on the oracle's reading
of gravity_hyperbolic.f90.  This test checks the discretisation itself: with
the density of the n = 1 polytrope (G = 1, unit radius) held fixed, the
potential the hyperbolic sub-cycles relax towards (psi -> 0 makes the
discrete Laplacian of phi equal 4 pi G rho, gravity_hyperbolic.f90:61-125)
must approach the analytic
    phi = -(4/pi) (1 + sin(pi r)/(pi r))  for r < 1,   -4/(pi r) outside,
at second order in the cell width: each halving of the width cuts the L1
error by about four (measured 4.7-5.1).  The grids are compared at the same
physical relaxation time (sub-cycle calls in proportion to the cell count
per axis), starting from the analytic potential.  A misread Laplacian
coefficient or Robin image would leave an error that does not shrink.

* Cartesian [-2, 2]^3 with the Robin condition phi ~ 1/r on every face,
  48^3, 96^3, 192^3;
* spherical (r, theta) with 4 theta cells, r in [0, 2], the coefficients of
  setup_grv_hyperbolic (gravity_hyperbolic.f90:336-405), 48, 96, 192
  radial cells."""
import numpy as np
import pytest

from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def relaxed_error(cfg, prims, phi_a, calls):
    """L1 of the potential against phi_a after `calls` gravity calls on the
    fixed density (each call: the CFL timestep of the unchanged state, then
    the hyperbolic sub-cycles of that dt)."""
    s = Simulation(cfg, prims, grvphi=phi_a)
    t, tn = s.time, 1
    for _ in range(calls):
        dt, _ = s.ctx.timestep(t, 1e30, 1e30)
        s.ctx.gravity_step(t, dt, tn)
        t, tn = t + dt, tn + 1
    phi = s.state(gravity=True)["grvphi"]
    s.close()
    return float(np.sum(np.abs(phi - phi_a)) / np.sum(np.abs(phi_a)))


@pytest.mark.parametrize("kind", ["cartesian", "spherical"])
def test_relaxed_potential_converges_at_second_order(kind):
    err = {}
    for n in (48, 96, 192):
        if kind == "cartesian":
            cfg, prims, phi = cases.polytrope(n)
        else:
            cfg, prims, phi = cases.polytrope_spherical((n, 4, 1))
        err[n] = relaxed_error(cfg, prims, phi, 200 * n // 48)
    print(kind, err)
    assert err[48] / err[96] > 3.5 and err[96] / err[192] > 3.5, err
    assert err[192] < 2e-4, err
