"""Slab decomposition along z on one GPU: the slabs of one grid, each its
own context, exchanging halos by device copies (hormone_b200.slab.
LocalExchange), give bit for bit the undecomposed run's state and dt,
periodic or not, with scalars, and in the mixed-precision form; so do
slabs whose stage kernels push their boundary layers into the neighbours'
halo buffers (mode "push"), and slabs with hyperbolic self-gravity, which
also exchange the potential's boundary layers."""
import numpy as np
import pytest

from hormone_b200 import slab
from hormone_b200.sim import Simulation

import cases

pytestmark = pytest.mark.gpu


def run_both(cfg, prims, world, steps, precision=0, mode="copy", grvphi=None):
    gravity = cfg["gravswitch"] == 3
    ref = Simulation(cfg, prims, precision=precision, grvphi=grvphi)
    dec = slab.LocalExchange(cfg, prims, world, precision=precision, mode=mode, grvphi=grvphi)
    for n in range(steps):
        ref.step()
        dec.step()
        for s in dec.ranks:
            assert s.dt == ref.dt, (n, s.dt, ref.dt)
    a, b = ref.state(gravity=gravity), dec.state()
    ref.close()
    dec.close()
    for k in a:
        assert a[k].shape == b[k].shape, k
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("world", [2, 3])
def test_orszag_tang_3d_periodic(world):
    cfg, prims = cases.ot3d(16)
    run_both(cfg, prims, world, 5)


def test_blast_reflective_three_slabs():
    cfg, prims = cases.blast3d(14, bc=1, mag=True)
    run_both(cfg, prims, 3, 5)


def test_spherical_phi_wedges():
    """A spherical polar grid (crdnt=2) split along phi into two wedges: the
    metric factors ride with the r and theta axes of every slab."""
    cfg, prims = cases.spherical((16, 12, 8), mag=True, xi1s=0.2)
    run_both(cfg, prims, 2, 5)


def test_cylindrical_z_slabs():
    """An axisymmetric cylindrical grid (R, z) split along z into three
    slabs, with periodic z."""
    cfg, prims = cases.cylindrical((24, 1, 18), mag=True)
    run_both(cfg, prims, 3, 5)


def test_riemann_with_scalars():
    cfg, prims = cases.riemann3d(n=(12, 10, 8), bc=(3, 1, 0), nspc=2)
    run_both(cfg, prims, 2, 5)


def test_mixed_precision_slabs():
    cfg, prims = cases.ot3d(16)
    run_both(cfg, prims, 2, 4, precision=1)


@pytest.mark.parametrize("world", [2, 3])
def test_polytrope_self_gravity_slabs(world):
    """Hyperbolic self-gravity on slabs: the potential's boundary layer is
    exchanged before every sub-stage of the sub-cycles and once more for
    the force of the hydro stages; the potential, psi and the state match
    the undecomposed run bit for bit."""
    cfg, prims, phi = cases.polytrope(16)
    run_both(cfg, prims, world, 4, grvphi=phi)


def test_self_gravity_slabs_stretched_z():
    """A z mesh of growing widths: each slab's own dtg_unit differs, the
    grid's is the minimum over the slabs."""
    cfg, prims, phi = cases.polytrope_stretched(16)
    dec = slab.LocalExchange(cfg, prims, 2, grvphi=phi)
    units = [s.ctx.gravity_unit() for s in dec.ranks]
    dec.close()
    assert units[0] == units[1]
    run_both(cfg, prims, 2, 4, grvphi=phi)


def test_self_gravity_slabs_mixed_precision():
    cfg, prims, phi = cases.polytrope(16)
    run_both(cfg, prims, 2, 3, precision=1, grvphi=phi)


@pytest.mark.parametrize("make", [lambda: cases.ot3d(16) + (None,), lambda: cases.polytrope(16)])
def test_evo_totals_over_slabs(make):
    """The evo_output totals summed over 3 slabs equal the undecomposed
    grid's to rounding (both sum per block; the slabs add their totals)."""
    cfg, prims, phi = make()
    ref = Simulation(cfg, prims, grvphi=phi)
    dec = slab.LocalExchange(cfg, prims, 3, grvphi=phi)
    for _ in range(3):
        ref.step()
        dec.step()
    a, b = ref.ctx.evo(), dec.evo()
    ref.close()
    dec.close()
    for k in a:
        assert abs(a[k] - b[k]) <= 1e-12 * max(abs(a[k]), 1e-300) + 1e-14 * abs(a["Etot"]), (k, a[k], b[k])


@pytest.mark.parametrize("world", [1, 2, 3])
def test_push_exchange_orszag_tang_periodic(world):
    """One slab wraps onto itself; two periodic slabs are each other's low
    and high neighbour."""
    cfg, prims = cases.ot3d(16)
    run_both(cfg, prims, world, 5, mode="push")


def test_push_exchange_blast_reflective():
    cfg, prims = cases.blast3d(14, bc=1, mag=True)
    run_both(cfg, prims, 3, 5, mode="push")


@pytest.mark.parametrize("nspc", [2, 5])
def test_push_exchange_with_scalars(nspc):
    """Scalar planes ride in the pushed layers (the 4- and 8-scalar
    kernels)."""
    cfg, prims = cases.riemann3d(n=(12, 10, 8), bc=(3, 1, 0), nspc=nspc)
    run_both(cfg, prims, 2, 5, mode="push")


@pytest.mark.parametrize("case", ["ot3d", "blast"])
def test_push_exchange_mixed_precision(case):
    if case == "ot3d":
        cfg, prims = cases.ot3d(16)
    else:
        cfg, prims = cases.blast3d(14, bc=1, mag=True)
    run_both(cfg, prims, 3, 4, precision=1, mode="push")


def test_push_exchange_refuses_curvilinear_and_gravity():
    from hormone_b200 import capi

    cfg, prims = cases.spherical((16, 12, 8), mag=True, xi1s=0.2)
    with pytest.raises(capi.HmnError):
        slab.LocalExchange(cfg, prims, 2, mode="push")


def test_decomposed_context_refuses_the_undecomposed_calls():
    cfg, prims = cases.ot3d(16)
    dec = slab.LocalExchange(cfg, prims, 2)
    from hormone_b200 import capi

    with pytest.raises(capi.HmnError):
        dec.ranks[0].ctx.hydro_step()
    with pytest.raises(capi.HmnError):
        dec.ranks[0].ctx.timestep(0.0, 1.0, 1.0)
    dec.close()


def test_distributed_step_on_one_rank_over_nccl():
    """The torch.distributed driver (NCCL all-reduce of the CFL partials
    viewed in place, collectives ordered on the slab's stream) on a
    one-rank group: the same bits as the undecomposed run."""
    dist = _one_rank_nccl()
    try:
        cfg, prims = cases.blast3d(14, bc=2, mag=True)
        ref = Simulation(cfg, prims)
        sim = slab.SlabSimulation(cfg, prims, 0, cfg["n"][2])
        ex = slab.TorchExchange(dist, 0, 1, periodic=False)
        sim.connect(False, False)
        for _ in range(4):
            ref.step()
            slab.run_distributed_step(sim, ex)
            assert sim.dt == ref.dt
        a, b = ref.state(), sim.state()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        ref.close()
        sim.close()
    finally:
        dist.destroy_process_group()


def _one_rank_nccl():
    import datetime
    import os
    import socket

    import torch
    import torch.distributed as dist

    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    return dist


def test_distributed_gravity_step_on_one_rank_over_nccl():
    """The distributed driver with self-gravity (the grid's dtg_unit shared
    by an all-reduce, the potential exchanged between sub-stages) on a
    one-rank group: the undecomposed run's bits."""
    dist = _one_rank_nccl()
    try:
        cfg, prims, phi = cases.polytrope(16)
        ref = Simulation(cfg, prims, grvphi=phi)
        sim = slab.SlabSimulation(cfg, prims, 0, cfg["n"][2], grvphi=phi)
        ex = slab.TorchExchange(dist, 0, 1, periodic=False)
        sim.connect(False, False)
        slab.share_gravity_unit(sim, ex)
        for _ in range(4):
            ref.step()
            slab.run_distributed_step(sim, ex)
            assert sim.dt == ref.dt
        assert ex.evo(sim) == sim.ctx.evo()  # one rank: the sum is its own totals
        a, b = ref.state(gravity=True), sim.state()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        ref.close()
        sim.close()
    finally:
        dist.destroy_process_group()


def test_symmetric_push_step_on_one_rank():
    """The push exchange's symmetric-memory buffers and step driver on a
    one-rank group (a periodic grid in one slab wraps onto itself, so no
    peer stores happen; several ranks need several GPUs)."""
    dist = _one_rank_nccl()
    try:
        cfg, prims = cases.ot3d(16)
        ref = Simulation(cfg, prims)
        sim = slab.SlabSimulation(cfg, prims, 0, cfg["n"][2], mode="push")
        halos = slab.SymmetricHalos(sim.halo_n)
        assert halos.peer(0, "hi", 1) == halos.local("hi", 1).data_ptr()
        slab.connect_symmetric(sim, halos, 0, 1, periodic=True)
        ex = slab.TorchExchange(dist, 0, 1, periodic=True)
        for _ in range(4):
            ref.step()
            slab.run_distributed_push_step(sim, ex)
            assert sim.dt == ref.dt
        a, b = ref.state(), sim.state()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        ref.close()
        sim.close()
    finally:
        dist.destroy_process_group()
