"""The benchmark configurations themselves on the GPU against the oracle, bit
for bit, in the reference's step order (hormone.f90:124-179: timestep,
gravity, hydro_step, phidamp):

* the Brio-Wu shock tube, 1024 cells on [0, 1], gamma = 2, Bx = 0.75,
  minmod, CFL 0.4, run to t = 0.1: dt of every step, the whole state every
  100 steps and at the end;
* the 3-D Orszag-Tang vortex on 256^3 with its seeded noise on vz and Bz:
  one full step (dt, ch, every conserved and primitive plane);
* the n = 1 polytrope with hyperbolic self-gravity on a 192^3 box
  [-2, 2]^3: three steps, with the potential and its time derivative;
* a 512^2 Kelvin-Helmholtz box advanced for three steps inside a batch of
  uneven boxes (persistent launches), against the oracle running it alone.

The oracle needs about 12 GB of host memory for the 256^3 grid and a few
seconds per step on the GPU host's cores."""
import numpy as np
import pytest

from hormone_b200 import config, grid as G, ic
from hormone_b200.batch import Batch, footprint
from oracle.oracle import Oracle

import cases
from test_gpu_parity import PRIMS, run_pair

pytestmark = pytest.mark.gpu


def test_brio_wu_1024_cells_to_t01():
    # the test set-ups count time in ms (dt_unit), so t = 0.1 is t_end = 100
    cfg = config.resolve("briowushock_x test", overrides=dict(ie=1024, t_end=100.0, dt_out=100.0, courant=0.4,
                                                              flux_limiter="minmod"))
    assert cfg["gamma"] == 2.0 and cfg["t_end"] == 0.1
    prims = ic.make(cfg, G.make_grid(cfg))
    o, s = run_pair(cfg, prims, 100000, check_every=100)
    assert s.time == o.scalars()["time"] and s.time >= 0.1 - 1e-15
    assert s.tn > 100


def test_orszag_tang_256_cubed_one_step():
    cfg, prims = cases.ot3d(256)
    o, s = run_pair(cfg, prims, 1)
    assert s.tn == 1 and s.ch == o.scalars()["ch"]


def test_polytrope_192_cubed_three_steps():
    cfg, prims, phi = cases.polytrope(192)
    o, s = run_pair(cfg, prims, 3, grvphi=phi)
    assert s.tn == 3


def test_kelvin_helmholtz_512_squared_inside_an_uneven_batch():
    rng = np.random.Generator(np.random.PCG64(20261203))
    boxes = []
    for n in (512, 131, 256, 300, 177):
        ratio, bx = float(rng.uniform(1, 4)), float(rng.uniform(0, 0.1))
        cfg, prims = cases.kh2d(n, ratio=ratio, bx=bx)
        boxes.append((cfg, prims))
    b = Batch(sum(footprint(c) for c, _ in boxes) + (1 << 24), max_sims=8, precision=0)
    slots = [b.add(c, p) for c, p in boxes]
    assert None not in slots
    b.step(3)
    t, tn, done, err = b.poll()
    got = b.download(slots[0])
    b.close()
    assert tn[slots[0]] == 3 and err[slots[0]] == 0
    cfg, prims = boxes[0]
    o = Oracle(cfg)
    o.set_prims(prims)
    o.start()
    for _ in range(3):
        o.step()
    assert t[slots[0]] == o.scalars()["time"]
    ou = o.u()
    for q in range(ou.shape[0]):
        assert np.array_equal(got["u"][q], ou[q]), q
    for k in PRIMS:
        assert np.array_equal(got[k], o.get(k)), k
