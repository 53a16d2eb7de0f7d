"""One grid decomposed into slabs along z, one slab per GPU.

This is the role of the reference's MPI domain decomposition
(src/main/mpi_domain.F90:256-339) for this path.  A rank owns the layers
[k0, k1) of the global grid.  Before every RK stage it exchanges the two
boundary layers of each primitive plane with its z neighbours; that is the
only data exchange of the step.  The CFL timestep is the all-reduced
minimum of the per-slab reductions (timestep.f90:56,87).  A slab's result is
bit-identical to the same cells of the undecomposed run: every cell sees the
same neighbours and the same operation order, and min/max reductions are
exact.

Two ways to move the halos:

- copy: before every stage each slab packs its boundary layers
  (``hmn_pack_halos``) and the exchange delivers them to the neighbours'
  halo buffers.  ``TorchExchange`` does it with point-to-point messages over
  ``torch.distributed`` (NCCL with CUDA tensors, gloo with CPU tensors for
  the host-side tests); ``LocalExchange`` with device copies.
- push (``hmn_set_slab_push``): each stage's kernel stores its boundary
  layers straight into the neighbours' halo buffers as it writes them
  (double-buffered by stage parity); between stages only a barrier runs.
  ``LocalExchange(mode="push")`` runs it with all slabs in one process;
  ``SymmetricHalos`` allocates the halo buffers in symmetric memory so that
  one process per GPU can store into its neighbours' buffers.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import capi, grid as gridmod, ic

PRIMS = ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")


def partition(nz: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous slabs [k0, k1) of as equal size as possible; each needs at
    least 2 layers (the stencil's reach)."""
    if world < 1 or nz < 2 * world:
        raise ValueError(f"cannot split {nz} layers into {world} slabs of at least 2")
    base, extra = divmod(nz, world)
    out, k = [], 0
    for r in range(world):
        size = base + (1 if r < extra else 0)
        out.append((k, k + size))
        k += size
    return out


def neighbours(rank: int, world: int, periodic: bool) -> Tuple[Optional[int], Optional[int]]:
    """Ranks of the lower and upper z neighbours (None at a physical face)."""
    lo = rank - 1 if rank > 0 else (world - 1 if periodic and world > 1 else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic and world > 1 else None)
    return lo, hi


def push_links(world: int, periodic: bool) -> List[Dict[str, Optional[Tuple[int, str]]]]:
    """For each rank of the push exchange: whose halo buffer its bottom
    layers go to (the low neighbour's "hi" buffers) and its top layers
    (the high neighbour's "lo" buffers); None on a physical face."""
    out = []
    for r in range(world):
        lo, hi = neighbours(r, world, periodic)
        out.append({"lo": None if lo is None else (lo, "hi"), "hi": None if hi is None else (hi, "lo")})
    return out


def slab_config(cfg: dict, k0: int, k1: int) -> dict:
    """The configuration of the slab [k0, k1): same settings, n[2] = k1 - k0."""
    c = dict(cfg)
    c["n"] = [cfg["n"][0], cfg["n"][1], k1 - k0]
    c["ke"] = c["ks"] + (k1 - k0) - 1 if "ks" in c else k1 - k0
    return c


def slab_grid(grid, k0: int, k1: int):
    """The global grid's z arrays restricted to the slab and its two ghost
    layers on each side (they are the neighbours' cells)."""
    out = [dict(grid[0]), dict(grid[1]), {}]
    for key, arr in grid[2].items():
        out[2][key] = np.ascontiguousarray(arr[k0:k1 + 4]) if isinstance(arr, np.ndarray) and arr.ndim == 1 else arr
    return out


class _DeviceArray:
    """A device pointer exposed through __cuda_array_interface__ (for
    torch.as_tensor views of memory the library owns)."""

    def __init__(self, ptr: int, n: int, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 2}


class SlabSimulation:
    """One rank's slab: the step of src/main/hormone.f90:126-155 split into the
    phases that the exchange interleaves."""

    def __init__(self, cfg: dict, prims_global: Dict[str, np.ndarray], k0: int, k1: int, precision: int = 0,
                 halo_alloc=None, local: bool = False, mode: str = "copy", grvphi=None, grvpsi=None,
                 cgrav_old: float = 0.0):
        """prims_global: the global primitives (sliced here), or with
        local=True the slab's own primitives (grvphi/grvpsi likewise, for
        self-gravity).  mode "copy" allocates send and receive halo buffers,
        "push" two receive buffers per face (one per stage parity)."""
        import torch

        self.cfg_global = cfg
        self.k0, self.k1 = k0, k1
        self.cfg = slab_config(cfg, k0, k1)
        self.grid = slab_grid(gridmod.make_grid(cfg), k0, k1)
        if local:
            local = prims_global
        else:
            local = {k: (v[..., k0:k1, :, :] if k == "spc" else v[k0:k1]) for k, v in prims_global.items()}
            grvphi = None if grvphi is None else np.ascontiguousarray(grvphi[k0:k1])
            grvpsi = None if grvpsi is None else np.ascontiguousarray(grvpsi[k0:k1])
        st = ic.to_state(self.cfg, local)
        self.ctx = capi.SlabContext(self.cfg, self.grid, precision=precision)
        self.ctx.upload(u=st["u"], prim=list(st["prim"]), grvphi=grvphi, grvpsi=grvpsi)
        self.nspc = int(self.cfg.get("nspc", 0))
        if self.nspc:
            self.ctx.upload_scalars(st["spc"])
        n = self.ctx.halo_bytes() // 8
        self.halo_n = n
        self.mode = mode
        alloc = halo_alloc or (lambda m: torch.zeros(m, dtype=torch.float64, device="cuda"))
        if mode == "push":
            self.recv = {(side, q): alloc(n) for side in ("lo", "hi") for q in (0, 1)}
        else:
            self.send_lo, self.send_hi, self.recv_lo, self.recv_hi = (alloc(n) for _ in range(4))
        self.gravity = cfg["gravswitch"] == 3
        if self.gravity:  # one layer of the potential per face
            self.ctx.set_gravity_clock(0.0, cgrav_old)
            m = self.ctx.gravity_halo_bytes() // 8
            self.gsend_lo, self.gsend_hi, self.grecv_lo, self.grecv_hi = (alloc(m) for _ in range(4))
        self.time, self.tn = 0.0, 0
        self.t_out, self.t_end = cfg["t_out"], cfg["t_end"]
        self.dt = self.ch = 0.0
        self.mag_glm = bool(cfg["mag_on"]) and cfg["dim"] > 1
        pmin, pmax = self.ctx.cfl_partials()
        self.cfl_min = torch.as_tensor(_DeviceArray(pmin, 1), device="cuda")
        self.cfl_max = torch.as_tensor(_DeviceArray(pmax, 1), device="cuda")

    def connect(self, has_lo: bool, has_hi: bool, wrap_lo: bool = False, wrap_hi: bool = False):
        """Attach the halo buffers; wrap_* mark faces that are the grid's
        periodic z boundary (first slab low, last slab high)."""
        p = lambda t: t.data_ptr()  # noqa: E731
        self.ctx.set_slab(p(self.send_lo) if has_lo else 0, p(self.send_hi) if has_hi else 0,
                          p(self.recv_lo) if has_lo else 0, p(self.recv_hi) if has_hi else 0, wrap_lo, wrap_hi)
        if self.gravity:
            self.ctx.set_slab_gravity(p(self.gsend_lo) if has_lo else 0, p(self.gsend_hi) if has_hi else 0,
                                      p(self.grecv_lo) if has_lo else 0, p(self.grecv_hi) if has_hi else 0)

    def connect_push(self, has_lo: bool, has_hi: bool, push_lo, push_hi, wrap_lo: bool = False,
                     wrap_hi: bool = False):
        """The push exchange: push_lo/push_hi are the (parity 0, parity 1)
        device addresses of the neighbours' buffers this slab stores into."""
        p = lambda t: t.data_ptr()  # noqa: E731
        rl = (p(self.recv["lo", 0]), p(self.recv["lo", 1])) if has_lo else (0, 0)
        rh = (p(self.recv["hi", 0]), p(self.recv["hi", 1])) if has_hi else (0, 0)
        self.ctx.set_slab_push(rl, rh, push_lo if has_lo else (0, 0), push_hi if has_hi else (0, 0), wrap_lo, wrap_hi)

    def stream(self):
        import torch

        return torch.cuda.ExternalStream(self.ctx.stream_ptr())

    # phases of one step
    def cfl_local(self):
        self.ctx.cfl_local(self.time, self.t_out, self.t_end)

    def cfl_finalize(self):
        self.dt, self.ch = self.ctx.cfl_finalize()

    def finish_step(self) -> bool:
        if self.mag_glm:
            self.ctx.phidamp()
        self.time = self.time + self.dt
        self.tn += 1
        c = self.cfg
        if c["endstyle"] == 1 and self.time >= self.t_end:
            return True
        if c["endstyle"] == 2 and self.tn >= c["tnlim"]:
            return True
        if c["outstyle"] == 1 and self.time >= self.t_out:
            self.t_out = self.t_out + c["dt_out"]
        return False

    def state(self) -> Dict[str, np.ndarray]:
        out = self.ctx.download(gravity=self.gravity)
        if self.nspc:
            out["spc"] = self.ctx.download_scalars()
        return out

    def close(self):
        self.ctx.close()


class LocalExchange:
    """All slabs of a grid in one process (e.g. on one GPU): halos move by
    device copies, the CFL partials by an in-process min/max."""

    def __init__(self, cfg: dict, prims: Dict[str, np.ndarray], world: int, precision: int = 0,
                 mode: str = "copy", grvphi=None, grvpsi=None, cgrav_old: float = 0.0):
        self.periodic = int(cfg["bc"][2][0][0]) == 0
        self.mode = mode
        self.parts = partition(cfg["n"][2], world)
        self.ranks = [SlabSimulation(cfg, prims, k0, k1, precision, mode=mode, grvphi=grvphi, grvpsi=grvpsi,
                                     cgrav_old=cgrav_old) for k0, k1 in self.parts]
        self.nb = [neighbours(r, world, self.periodic) for r in range(world)]
        self.gravity = self.ranks[0].gravity
        if mode == "push":
            links = push_links(world, self.periodic)
            for r, s in enumerate(self.ranks):
                lo, hi = self.nb[r]
                tgt = {}
                for face in ("lo", "hi"):
                    link = links[r][face]
                    tgt[face] = ((0, 0) if link is None else
                                 tuple(self.ranks[link[0]].recv[link[1], q].data_ptr() for q in (0, 1)))
                s.connect_push(lo is not None, hi is not None, tgt["lo"], tgt["hi"], wrap_lo=r == 0,
                               wrap_hi=r == world - 1)
            for s in self.ranks:  # the initial state's boundary layers
                s.ctx.pack_halos()
            self._sync()
            return
        for r, s in enumerate(self.ranks):
            lo, hi = self.nb[r]
            s.connect(lo is not None, hi is not None, wrap_lo=r == 0, wrap_hi=r == world - 1)
        if self.gravity:  # the grid's dtg_unit: the minimum over the slabs
            unit = min(s.ctx.gravity_unit() for s in self.ranks)
            for s in self.ranks:
                s.ctx.set_gravity_unit(unit)

    def _exchange_gravity(self):
        """The potential's boundary layers to the neighbours' halos."""
        import torch

        for s in self.ranks:
            s.ctx.pack_gravity_halos()
        self._sync()
        for r, s in enumerate(self.ranks):
            lo, hi = self.nb[r]
            if lo is not None:
                s.grecv_lo.copy_(self.ranks[lo].gsend_hi)
            if hi is not None:
                s.grecv_hi.copy_(self.ranks[hi].gsend_lo)
        torch.cuda.synchronize()

    def _sync(self):
        import torch

        for s in self.ranks:
            s.ctx.sync()
        torch.cuda.synchronize()

    def step(self) -> bool:
        import torch

        for s in self.ranks:
            s.cfl_local()
        self._sync()
        gmin = torch.min(torch.cat([s.cfl_min for s in self.ranks]))
        gmax = torch.max(torch.cat([s.cfl_max for s in self.ranks]))
        for s in self.ranks:
            s.cfl_min.copy_(gmin.reshape(1))
            s.cfl_max.copy_(gmax.reshape(1))
        torch.cuda.synchronize()
        for s in self.ranks:
            s.cfl_finalize()
        if self.gravity:  # gravity.f90 sub-stages, each after an exchange of the potential
            nsub = {s.ctx.gravity_begin(s.time, s.dt, s.tn) for s in self.ranks}
            assert len(nsub) == 1, nsub
            for _ in range(nsub.pop()):
                self._exchange_gravity()
                for s in self.ranks:
                    s.ctx.gravity_substage()
            self._exchange_gravity()  # the force of the hydro stages
        for stage in range(1, self.cfg_rk() + 1):
            if self.mode == "push":  # the previous stage of every slab has stored its layers
                self._sync()
                for s in self.ranks:
                    s.ctx.hydro_stage(stage)
                continue
            for s in self.ranks:
                s.ctx.pack_halos()
            self._sync()
            for r, s in enumerate(self.ranks):
                lo, hi = self.nb[r]
                if lo is not None:
                    s.recv_lo.copy_(self.ranks[lo].send_hi)
                if hi is not None:
                    s.recv_hi.copy_(self.ranks[hi].send_lo)
            torch.cuda.synchronize()
            for s in self.ranks:
                s.ctx.hydro_stage(stage)
        ends = [s.finish_step() for s in self.ranks]
        return ends[0]

    def cfg_rk(self) -> int:
        return int(self.ranks[0].cfg["rktype"])

    def evo(self) -> Dict[str, float]:
        """The evo_output totals of the whole grid: each slab's hmn_evo
        totals added in slab order (output.f90:235-244 all-reduces them)."""
        out: Dict[str, float] = {}
        for s in self.ranks:
            for k, v in s.ctx.evo().items():
                out[k] = out.get(k, 0.0) + v
        return out

    def state(self) -> Dict[str, np.ndarray]:
        """The global state assembled from the slabs (z is the slowest axis)."""
        parts = [s.state() for s in self.ranks]
        out = {}
        for k in parts[0]:
            axis = 1 if parts[0][k].ndim == 4 else 0
            out[k] = np.concatenate([p[k] for p in parts], axis=axis)
        return out

    def close(self):
        for s in self.ranks:
            s.close()


class TorchExchange:
    """One slab per process over torch.distributed (NCCL on GPUs, gloo for
    CPU tensors).  Every rank posts its sends high-then-low and its receives
    low-then-high, so with two periodic ranks (both neighbours the same
    peer) the messages still pair up face to face."""

    def __init__(self, dist, rank: int, world: int, periodic: bool):
        self.dist, self.rank, self.world = dist, rank, world
        self.lo, self.hi = neighbours(rank, world, periodic)

    def halos(self, send_lo, send_hi, recv_lo, recv_hi):
        d = self.dist
        ops = []
        if self.hi is not None:
            ops.append(d.P2POp(d.isend, send_hi, self.hi))
        if self.lo is not None:
            ops.append(d.P2POp(d.isend, send_lo, self.lo))
        if self.lo is not None:
            ops.append(d.P2POp(d.irecv, recv_lo, self.lo))
        if self.hi is not None:
            ops.append(d.P2POp(d.irecv, recv_hi, self.hi))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()

    def cfl(self, tmin, tmax):
        self.dist.all_reduce(tmin, op=self.dist.ReduceOp.MIN)
        self.dist.all_reduce(tmax, op=self.dist.ReduceOp.MAX)

    def evo(self, sim: "SlabSimulation") -> Dict[str, float]:
        """The evo_output totals of the whole grid: this slab's hmn_evo
        totals summed over the ranks (output.f90:235-244)."""
        import torch

        tot = sim.ctx.evo()
        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([tot[k] for k in tot], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return dict(zip(tot, t.tolist()))

    def min_scalar(self, v: float) -> float:
        """The minimum of a host double over the ranks."""
        import torch

        dev = "cuda" if self.dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        return float(t.item())


def share_gravity_unit(sim: "SlabSimulation", ex: TorchExchange):
    """Every rank's dtg_unit becomes the grid's (the minimum over slabs)."""
    if sim.gravity:
        sim.ctx.set_gravity_unit(ex.min_scalar(sim.ctx.gravity_unit()))


class SymmetricHalos:
    """The push exchange's halo buffers in symmetric memory, one process per
    GPU: a rank's four receive buffers (low and high face, two stage
    parities) are one symmetric allocation, so a neighbour's kernel can
    store into them directly (peer access over NVLink).  Sections are
    ordered (lo, 0), (lo, 1), (hi, 0), (hi, 1) of ``n`` doubles each.
    (Exercised on a one-rank group only; peer stores between GPUs are
    untested.)"""

    SECTION = {("lo", 0): 0, ("lo", 1): 1, ("hi", 0): 2, ("hi", 1): 3}

    def __init__(self, n: int, group=None):
        import torch
        import torch.distributed as dist
        import torch.distributed._symmetric_memory as symm_mem

        self.n = n
        self.buf = symm_mem.empty(4 * n, dtype=torch.float64, device="cuda")
        self.buf.zero_()
        self.hdl = symm_mem.rendezvous(self.buf, group if group is not None else dist.group.WORLD)
        ptrs = self.hdl.buffer_ptrs
        self.ptrs = list(ptrs() if callable(ptrs) else ptrs)

    def local(self, side: str, q: int):
        k = self.SECTION[side, q]
        return self.buf[k * self.n:(k + 1) * self.n]

    def peer(self, rank: int, side: str, q: int) -> int:
        """Device address of rank's (side, parity) buffer in this process."""
        return int(self.ptrs[rank]) + self.SECTION[side, q] * self.n * 8


def connect_symmetric(sim: "SlabSimulation", halos: SymmetricHalos, rank: int, world: int, periodic: bool):
    """Wire a push-mode slab to its neighbours' symmetric halo buffers and
    store the initial boundary layers (followed by the caller's barrier)."""
    links = push_links(world, periodic)[rank]
    lo, hi = neighbours(rank, world, periodic)
    sim.recv = {(side, q): halos.local(side, q) for side in ("lo", "hi") for q in (0, 1)}
    tgt = {face: ((0, 0) if links[face] is None else
                  tuple(halos.peer(links[face][0], links[face][1], q) for q in (0, 1))) for face in ("lo", "hi")}
    sim.connect_push(lo is not None, hi is not None, tgt["lo"], tgt["hi"], wrap_lo=rank == 0,
                     wrap_hi=rank == world - 1)
    sim.ctx.pack_halos()


def run_distributed_push_step(sim: "SlabSimulation", ex: TorchExchange) -> bool:
    """One step of one rank with the push exchange: the CFL all-reduce, then
    per stage a barrier (every slab finished the previous stage, so its
    layers are in place) and the stage, whose kernel stores this slab's
    boundary layers into the neighbours' buffers."""
    import torch

    with torch.cuda.stream(sim.stream()):
        sim.cfl_local()
        ex.cfl(sim.cfl_min, sim.cfl_max)
        sim.cfl_finalize()
        for stage in range(1, int(sim.cfg["rktype"]) + 1):
            sim.ctx.sync()
            ex.dist.barrier()
            sim.ctx.hydro_stage(stage)
    return sim.finish_step()


def run_distributed_step(sim: SlabSimulation, ex: TorchExchange) -> bool:
    """One step of one rank, the collectives ordered on the slab's stream."""
    import torch

    with torch.cuda.stream(sim.stream()):
        sim.cfl_local()
        ex.cfl(sim.cfl_min, sim.cfl_max)
        sim.cfl_finalize()
        if sim.gravity:  # share_gravity_unit ran once before the first step
            for _ in range(sim.ctx.gravity_begin(sim.time, sim.dt, sim.tn)):
                sim.ctx.pack_gravity_halos()
                ex.halos(sim.gsend_lo, sim.gsend_hi, sim.grecv_lo, sim.grecv_hi)
                sim.ctx.gravity_substage()
            sim.ctx.pack_gravity_halos()
            ex.halos(sim.gsend_lo, sim.gsend_hi, sim.grecv_lo, sim.grecv_hi)
        for stage in range(1, int(sim.cfg["rktype"]) + 1):
            sim.ctx.pack_halos()
            ex.halos(sim.send_lo, sim.send_hi, sim.recv_lo, sim.recv_hi)
            sim.ctx.hydro_stage(stage)
    return sim.finish_step()
