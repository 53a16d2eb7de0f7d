#!/usr/bin/env python
"""Zone-updates/s of HORMONE's explicit MHD step on B200.

Workload: the 3-D Orszag-Tang-type vortex on a 256^3 periodic unit box
(gamma=5/3, modified_mc MUSCL + HLLD + GLM, SSP-RK3, courant 0.9, seeded
1e-3 noise on vz and Bz).  One step = timestep (CFL reduction) + three fused
RK stages + phidamp + time advance, i.e. one zone-update per cell per step.
The 1.2 GB state per RK buffer is far larger than the 126 MB L2, so no
flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W]          the CUDA path
  python bench.py --impl reference ...                      the CPU path

With N>1 (torchrun) every rank advances its own independent 256^3 box
(weak scaling, no data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "zone-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--cpu-size", type=int, default=0, help="edge of the box the CPU legs time (0: --size)")
    ap.add_argument("--cpu-steps", type=int, default=5)
    ap.add_argument("--no-extra", action="store_true", help="skip the compact kh_batch and serve legs")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--workload", choices=["ot3d", "kh-batch", "serve", "polytrope", "polytrope-sph", "briowu", "sedov"], default="ot3d",
                    help="ot3d: the headline (3-D Orszag-Tang 256^3); kh-batch: 512 uneven 2-D KH boxes batched vs "
                         "one at a time; serve: a Poisson request stream through the continuous-batching server; "
                         "polytrope: 192^3 self-gravitating polytrope with hyperbolic gravity")
    ap.add_argument("--boxes", type=int, default=512)
    ap.add_argument("--schedule", default="",
                    help="kh-batch: TILE,GRID,SWEEP for the 2-D kind instead of the autotuner's choice")
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--policy", choices=["fifo", "sjf", "priority"], default="priority",
                    help="serve admission and stepping order")
    ap.add_argument("--live-cells", type=int, default=0, help="serve: cap on the admitted cells (0: none)")
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--poly-steps", type=int, default=2000, help="timed steps of the polytrope workload")
    ap.add_argument("--decomp", choices=["replicas", "slab"], default="replicas",
                    help="ot3d with N>1: independent boxes per rank (default), or one periodic grid of "
                         "size x size x (size*N) split into z slabs with NCCL halo exchange")
    return ap.parse_args()


def ot_config(n, nz=None, zlen=1.0):
    from hormone_b200 import config

    return config.resolve("orszagtang_3d", overrides=dict(
        ie=n, je=n, ke=nz or n, xi3s=0.0, xi3e=zlen, mag_on=True, gamma=1.6666666666666667, courant=0.9,
        flux_limiter="modified_mc", t_end=0.5, dt_out=0.5))


def ot_prims(cfg, seed):
    from hormone_b200 import grid as G, ic

    return ic.orszagtang3d(cfg, G.make_grid(cfg), seed=seed)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profiled_value(key, prefix="stage_kernel_ot3d"):
    """A figure of a committed ncu summary (profiles/<prefix>*.md, a line
    '<key>: X'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if fn.startswith(prefix) and fn.endswith(".md"):
            m = re.search(re.escape(key) + r":\s*([0-9.eE+-]+)", open(os.path.join(pdir, fn)).read())
            if m:
                return float(m.group(1))
    return None


def profiled_traffic(prefix="stage_kernel_ot3d"):
    """DRAM bytes per cell of one stage launch (ncu dram__bytes_read.sum +
    dram__bytes_write.sum over the cells of the launch)."""
    return profiled_value("dram_bytes_per_cell", prefix)


def profile_source(prefix):
    """The committed ncu summary the profiled figures come from, and the
    commit of the kernel it captured (its line 'captured_at_commit: X')."""
    pdir = os.path.join(ROOT, "profiles")
    for fn in sorted(os.listdir(pdir)) if os.path.isdir(pdir) else []:
        if fn.startswith(prefix) and fn.endswith(".md"):
            m = re.search(r"captured_at_commit:\s*([0-9a-f]+)", open(os.path.join(pdir, fn)).read())
            return {"file": f"profiles/{fn}", "commit": m.group(1) if m else None}
    return None


def ot_line_config(n, world):
    """config of the Orszag-Tang line, the same for the GPU and the reference arm."""
    return {"workload": f"orszag-tang-3d-{n}^3-fp64", "grid": [n, n, n], "cells_per_gpu": n ** 3,
            "limiter": "modified_mc", "rktype": 3, "courant": 0.9,
            "l2": f"inputs larger than L2 (9 x 8 B x {n}^3 = {9 * 8 * n ** 3 / 1e9:.2f} GB per RK buffer)",
            "parallelism": f"replicas{world}"}


# ---------------------------------------------------------------------------
def cpu_leg(n, steps, warm=1):
    """The oracle (C restatement, OpenMP over all host cores) on an n^3 box of
    the same workload: zone-updates/s."""
    from oracle.oracle import Oracle

    cfg = ot_config(n)
    o = Oracle(cfg)
    o.set_prims(ot_prims(cfg, 20261203))
    o.start()
    for _ in range(warm):
        o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return n ** 3 * steps / dt, cores, dt


def run_reference(args, rank):
    if rank != 0:
        return
    import oracle.oracle as orc  # noqa: F401  (builds liboracle.so if needed)

    # the GPU arm's grid and workload; the CPU steps are the sample: at most
    # --steps of them (about 3 s each at 256^3 on 16 cores), one untimed
    n = args.size
    steps = max(3, min(args.steps, 20))
    from oracle.oracle import Oracle

    cfg = ot_config(n)
    o = Oracle(cfg)
    o.set_prims(ot_prims(cfg, 20261203))
    o.start()
    for _ in range(min(args.warmup, 1)):
        o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    v = n ** 3 * steps / el
    sample = (f"{n}^3 box of the same 3-D Orszag-Tang workload, {steps} full steps after {min(args.warmup, 1)} "
              f"untimed; CPU restatement of HORMONE's FP64 step (the Fortran reference cannot be compiled here), "
              f"OpenMP over {cores} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus,
            "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * el / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": ot_line_config(n, args.gpus),
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def mixed_leg(args, cfg, prims, sim64, rank, world, dist):
    """The FP32-flux / FP64-accumulate form on the same workload: throughput,
    and the one-step L1 error per variable against the FP64 form started
    from the same state (sum |q_mixed - q_fp64| / sum |q_fp64|)."""
    import numpy as np
    import torch

    from hormone_b200.sim import Simulation

    n = args.size
    sim = Simulation(cfg, prims, precision=1)
    stream = torch.cuda.ExternalStream(sim.ctx.stream_ptr())
    sim.run_device(max_steps=args.warmup)
    torch.cuda.synchronize()
    sim.ctx.sync()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    t, nrun = sim.ctx.run(sim.time, cfg["t_end"], args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = world * n ** 3 * nrun / (ms * 1e-3)
    # one step from an identical state
    st = sim64.state()
    prim = [st[k] for k in ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")]
    for s_ in (sim64, sim):
        s_.ctx.upload(u=st["u"], prim=prim)
        s_.time, s_.tn = 0.1, 1
    sim64.step()
    sim.step()
    a, b = sim64.state(), sim.state()
    l1 = {k: float(np.sum(np.abs(b[k] - a[k])) / max(np.sum(np.abs(a[k])), 1e-300))
          for k in ("d", "e", "v1", "v2", "v3", "b1", "b2", "b3")}
    sim.close()
    return {"value": value, "unit": METRIC, "ms_per_step": ms / max(nrun, 1), "steps": nrun,
            "dtype": "f32 Riemann solver / f64 reconstruction, pressure recovery and compensated accumulation",
            "l1_one_step_vs_fp64": l1, "vs_fp64_48^3_100_steps": mixed_accuracy(48, 100)}


def mixed_accuracy(n, steps):
    """The mixed form against the FP64 form (bit-identical to the oracle)
    on the same workload at n^3, both run to the time the FP64 form reaches
    in `steps` steps: per conserved variable sum |q - q64| dV / sum |q64| dV,
    and the max / L1 / L2 norms of HORMONE's test harness (tests.f90:46-292)
    with the FP64 state as the reference.  For scale, the same L1 of an FP64
    run whose initial primitives carry a relative perturbation of 1e-8 (the
    size of an FP32 rounding): the flow's own sensitivity."""
    import numpy as np

    from hormone_b200 import norms
    from hormone_b200.sim import Simulation

    cfg = ot_config(n)
    prims = ot_prims(cfg, 20261203)
    a = Simulation(cfg, prims)
    for _ in range(steps):
        a.step()
    b = Simulation(cfg, prims, precision=1)
    b.ctx.run(0.0, a.time, 10 * steps)
    rng = np.random.default_rng(7)
    pert = {k: (v * (1.0 + 1e-8 * rng.uniform(-1.0, 1.0, v.shape)) if k in ("d", "p", "v1", "v2", "v3") else v)
            for k, v in prims.items()}
    c = Simulation(cfg, pert)
    c.ctx.run(0.0, a.time, 10 * steps)
    sa, sb, sc = a.state(), b.state(), c.state()
    for s_ in (a, b, c):
        s_.close()
    names = ("d", "m1", "m2", "m3", "E", "b1", "b2", "b3", "phi")

    def l1(x):
        return {names[q]: float(np.sum(np.abs(x["u"][q] - sa["u"][q])) / max(np.sum(np.abs(sa["u"][q])), 1e-300))
                for q in range(sa["u"].shape[0])}

    tests_f90 = {k: {m: v[m] for m in ("max", "L1", "L2")} for k, v in norms.compare(sb, sa, cfg).items()}
    return {"t": a.time, "l1_conserved": l1(sb), "tests_f90_norms": tests_f90,
            "fp64_perturbed_1e-8_l1_conserved": l1(sc)}


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from hormone_b200 import ic
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist_

        dist = dist_
    n = args.size
    cfg = ot_config(n)
    prims = ot_prims(cfg, 20261203 + rank)
    sim = Simulation(cfg, prims)
    stream = torch.cuda.ExternalStream(sim.ctx.stream_ptr())
    cells = n ** 3

    def barrier():
        torch.cuda.synchronize()
        sim.ctx.sync()
        if dist:
            dist.barrier()

    # warm-up
    sim.run_device(max_steps=args.warmup)
    barrier()
    l0 = sim.ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        barrier()
        e0.record(stream)
        t_before = sim.time
        _, nrun = sim.ctx.run(sim.time, cfg["t_end"], args.steps)
        sim.time = _
        e1.record(stream)
        e1.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    launches = sim.ctx.launches() - l0
    if nrun != args.steps:
        raise RuntimeError(f"only {nrun} of {args.steps} steps ran (t_end reached)")
    if dist:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * cells * args.steps / (ms * 1e-3)
    clocks = clk.summary()

    # dominant kernel: the fused RK stage, timed per launch on its stream
    k = max(3, args.steps)
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    h0.record(stream)
    for _ in range(k):
        sim.ctx.hydro_step()
    h1.record(stream)
    h1.synchronize()
    stage_ms = h0.elapsed_time(h1) / (3 * k)
    nvar = cfg["nvar"]
    alg_bytes = (2 + 3 + 3) * nvar * 8 / 3 * cells  # per stage launch, averaged over the 3 stages
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9
    prof = "march_stage_ot3d"  # the ncu summary of the stage kernel this grid runs on
    tpc = profiled_traffic(prof)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": (tpc * cells) if tpc else None, "kernel": "march_stage_kernel",
                "alg_bytes_per_launch": alg_bytes, "launch_ms": stage_ms, "peak_kind": peak_kind,
                "traffic_source": profile_source(prof),
                "note": "FP64-issue-bound stencil: frac is of measured HBM copy bandwidth; the instruction "
                        "bounds below use per-cell instruction counts from the ncu summary in traffic_source "
                        "(counts per cell do not depend on timing) and this run's launch time and SM clock"}
    # the bounds the stage actually meets: issue slots (one warp instruction
    # per cycle per SM sub-partition) and the FP64 pipe (a warp instruction
    # takes it for two cycles: 16 FP64 lanes per sub-partition)
    winst, fpinst = profiled_value("warp_inst_per_cell", prof), profiled_value("fp64_warp_inst_per_cell", prof)
    nsm = torch.cuda.get_device_properties(local_rank).multi_processor_count
    clk_hz = (clocks.get("sm_mhz") or 1965.0) * 1e6
    slots = stage_ms * 1e-3 * nsm * 4 * clk_hz
    if winst:
        roofline["issue_frac"] = winst * cells / slots
    if fpinst:
        roofline["fp64_pipe_frac"] = 2 * fpinst * cells / slots

    # end to end through the drop-in C ABI with pinned host buffers: the
    # conserved state U goes up (hmn_upload derives the primitives from it on
    # the device, as `primitive` does), the steps run through the per-call
    # entry points, and the new U comes back
    e2e = None
    if not args.no_e2e and rank == 0:
        st = ic.to_state(cfg, prims)
        u_h = torch.empty(st["u"].shape, dtype=torch.float64, pin_memory=True).numpy()
        u_h[...] = st["u"]
        out_u = torch.empty(st["u"].shape, dtype=torch.float64, pin_memory=True).numpy()
        from hormone_b200 import capi

        ctx = sim.ctx
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.upload(u=u_h)
        t = 0.0
        for _ in range(args.steps):
            dt, ch = ctx.timestep(t, cfg["t_end"], cfg["t_end"])
            ctx.hydro_step()
            ctx.phidamp()
            t = t + dt
        rc = capi.lib().hmn_download(ctx.h, capi._dp(out_u), None, None, None)
        if rc != 0:
            raise capi.HmnError(rc, "hmn_download")
        el = time.perf_counter() - t0
        hb = u_h.nbytes + 24 * args.steps
        db = out_u.nbytes + 200 * args.steps
        e2e = {"value": cells * args.steps / el, "unit": METRIC, "h2d_bytes_per_step": hb / args.steps,
               "d2h_bytes_per_step": db / args.steps, "steps": args.steps,
               "path": "hmn_upload(U) + per step hmn_timestep/hmn_hydro_step/hmn_phidamp + hmn_download(U)"}

    mixed = None
    if not args.no_mixed:
        mixed = mixed_leg(args, cfg, prims, sim, rank, world, dist)

    sim.close()
    extra = {}
    if rank == 0 and world == 1 and not args.no_extra:
        extra = extra_legs(args, value, local_rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cn = args.cpu_size or n
        v, cores, el = cpu_leg(cn, args.cpu_steps)
        cpu = {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"{cn}^3 box of the same workload, {args.cpu_steps} full steps after one untimed "
                         f"({el:.1f} s) of the CPU restatement, OpenMP"}
    if rank == 0:
        config = ot_line_config(n, world)
        config["precision"] = "fp64 bit-compatible (no FMA)"
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "mixed": mixed,
                "clocks": clocks}
        line.update(extra)
        print(json.dumps(line), flush=True)


def kh_boxes(nboxes, seed=20261203):
    """(cfg, density ratio, Bx) of the periodic Kelvin-Helmholtz boxes of the
    batched benchmark: edges round(128 * 4^u), u ~ U[0, 1], seeded."""
    import numpy as np

    from hormone_b200 import config

    rng = np.random.Generator(np.random.PCG64(seed))
    boxes = []
    for _ in range(nboxes):
        n = int(round(128 * 4 ** rng.uniform()))
        ratio, bx = float(rng.uniform(1, 4)), float(rng.uniform(0, 0.1))
        ov = dict(ie=n, je=n, ke=1, mag_on=True, gamma=1.6666666666666667, t_end=2.0, dt_out=2.0,
                  xi1s=-0.5, xi1e=0.5, xi2s=-0.5, xi2e=0.5)
        boxes.append((config.resolve("kh_batch", overrides=ov), ratio, bx))
    return boxes


def batch_leg(boxes, steps, warmup, precision):
    """`steps` steps of every box in one batch (persistent launches, autotuned
    schedule, CUDA graph), timed on the batch's stream: zone-updates/s."""
    import numpy as np
    import torch

    from hormone_b200 import autotune
    from hormone_b200.batch import Batch, footprint

    sched = autotune.tune(boxes[:32], precision=precision, steps=2, cache=None)
    b = Batch(sum(footprint(c) for c, _ in boxes) + (1 << 26), max_sims=len(boxes) + 1, precision=precision)
    for c, p in boxes:
        assert b.add(c, p) is not None
    autotune.apply(b, sched)
    stream = torch.cuda.ExternalStream(b.stream_ptr())
    b.step(warmup)
    b.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    b.close()
    cells = sum(int(np.prod(c["n"])) for c, _ in boxes)
    return {"value": cells * steps / (ms * 1e-3), "ms_per_step": ms / steps, "cells": cells}


def extra_legs(args, plain_fp64, local_rank):
    """The batched and served forms on compact versions of their benchmarks,
    each in FP64 and in the mixed form, with the ratios of the mixed form to
    the plain FP64 form (the Orszag-Tang value of this line) and to the same
    form in FP64."""
    import torch

    from hormone_b200 import grid as G, ic, serve
    from hormone_b200.batch import Batch

    boxes = [(c, ic.kelvin_helmholtz(c, G.make_grid(c), r, bx)) for c, r, bx in kh_boxes(64)]
    kb = {p: batch_leg(boxes, 20, 3, p) for p in (0, 1)}
    kh = {"workload": "kh-batch-64-boxes-128^2..512^2: the first 64 boxes of the 512-box set, 20 steps after 3",
          "cells": kb[0]["cells"], "fp64": kb[0]["value"], "mixed": kb[1]["value"],
          "ms_per_step": {"fp64": kb[0]["ms_per_step"], "mixed": kb[1]["ms_per_step"]},
          "mixed_over_fp64_batch": kb[1]["value"] / kb[0]["value"],
          "mixed_over_plain_fp64": kb[1]["value"] / plain_fp64}
    sv = {}
    for p in (0, 1):
        reqs = serve.make_requests(32, rate=50.0, seed=20261203)
        free, _ = torch.cuda.mem_get_info()
        b = Batch(int(free * 0.6), max_sims=1024, precision=p)
        st = serve.serve(reqs, b, chunk=8, keep_results=False, policy="priority").summary()
        b.close()
        sv[p] = st
    srv = {"workload": "serve-32-requests-poisson-50/s: the first 32 requests of the seeded 4096-request stream",
           "fp64": {k: sv[0][k] for k in ("zone_updates_per_s", "p50_s", "p99_s", "completed", "failed")},
           "mixed": {k: sv[1][k] for k in ("zone_updates_per_s", "p50_s", "p99_s", "completed", "failed")},
           "mixed_over_fp64_served": sv[1]["zone_updates_per_s"] / sv[0]["zone_updates_per_s"],
           "mixed_over_plain_fp64": sv[1]["zone_updates_per_s"] / plain_fp64}
    return {"kh_batch": kh, "serve": srv}


def run_slab(args, rank, world, local_rank):
    """One periodic grid of n x n x (n*N) cells decomposed into N z slabs of
    n^3, one per rank: each step all-reduces the CFL partials and exchanges
    2-layer halos before every RK stage (NCCL).  The initial noise is seeded
    per slab."""
    import torch
    import torch.distributed as dist

    from hormone_b200 import grid as G, ic, slab

    torch.cuda.set_device(local_rank)
    n = args.size
    cfg = ot_config(n, nz=n * world, zlen=float(world))
    k0, k1 = slab.partition(n * world, world)[rank]
    lcfg = slab.slab_config(cfg, k0, k1)
    lgrid = slab.slab_grid(G.make_grid(cfg), k0, k1)
    prims = ic.orszagtang3d(lcfg, lgrid, seed=20261203 + rank)
    sim = slab.SlabSimulation(cfg, prims, k0, k1, local=True)
    ex = slab.TorchExchange(dist, rank, world, periodic=True)
    sim.connect(ex.lo is not None, ex.hi is not None, wrap_lo=rank == 0, wrap_hi=rank == world - 1)
    stream = sim.stream()
    for _ in range(args.warmup):
        slab.run_distributed_step(sim, ex)
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            slab.run_distributed_step(sim, ex)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        dist.barrier()
    t = torch.tensor([e0.elapsed_time(e1)], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    cells = n ** 3 * world
    sim.close()
    if rank == 0:
        line = {"metric": METRIC, "value": cells * args.steps / (ms * 1e-3), "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": f"orszag-tang-3d-{n}x{n}x{n * world}-fp64-slabs", "grid": [n, n, n * world],
                           "cells_per_gpu": n ** 3, "parallelism": f"z-slabs{world}",
                           "exchange": "NCCL 2-layer halos of the primitive planes before every RK stage, "
                                       "all-reduce min/max of the CFL partials"},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)


def run_kh_batch(args, rank=0, world=1, local_rank=0):
    """512 periodic KH boxes, edges round(128*4^u) with u ~ U[0,1] (seeded):
    K steps of every box in one batch (persistent launches, autotuned
    schedule, CUDA graph) against the same K steps box by box.  With N ranks
    the boxes are split by footprint (independent simulations, no
    collective); the time is the max over ranks."""
    import math

    import numpy as np
    import torch

    from hormone_b200 import autotune, config, grid as G, ic, shard
    from hormone_b200.batch import Batch, footprint
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

    boxes = kh_boxes(args.boxes)
    total_cells = sum(int(np.prod(c["n"])) for c, _, _ in boxes)
    mine = shard.my_share([footprint(c) for c, _, _ in boxes], rank, world)
    boxes = [(c, ic.kelvin_helmholtz(c, G.make_grid(c), r, b)) for i, (c, r, b) in enumerate(boxes) if i in set(mine)]
    cells = sum(int(np.prod(c["n"])) for c, _ in boxes)
    K = args.steps
    if args.schedule:
        sched = {1: tuple(int(x) for x in args.schedule.split(","))}
    else:
        sched = autotune.tune(boxes[:32], precision=args.precision, steps=2, cache=None)
    b = Batch(sum(footprint(c) for c, _ in boxes) + (1 << 26), max_sims=len(boxes) + 1, precision=args.precision)
    for c, p in boxes:
        assert b.add(c, p) is not None
    autotune.apply(b, sched)
    stream = torch.cuda.ExternalStream(b.stream_ptr())
    b.step(args.warmup)
    b.sync()
    if dist:
        dist.barrier()
    l0 = b.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        b.step(K)
        e1.record(stream)
        e1.synchronize()
    ms_b = shard.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
    launches_b = b.launches() - l0
    b.close()
    # one at a time: every box's K steps through its own context, box after box
    sims = [Simulation(c, p, precision=args.precision) for c, p in boxes]
    for s_ in sims:
        s_.run_device(max_steps=1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    l1 = sum(s_.ctx.launches() for s_ in sims)
    for s_ in sims:
        s_.ctx.run(s_.time, s_.t_end, K)
    for s_ in sims:
        s_.ctx.sync()
    ms_1 = shard.max_over_ranks((time.perf_counter() - t0) * 1e3, dist, device="cuda")
    launches_1 = sum(s_.ctx.launches() for s_ in sims) - l1
    for s_ in sims:
        s_.close()
    if rank != 0:
        return
    cells = total_cells
    line = {"metric": METRIC, "value": cells * K / (ms_b * 1e-3), "unit": METRIC, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_b / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "mixed", "data": "synthetic",
            "config": {"workload": f"kh-batch-{args.boxes}-boxes-128^2..512^2", "cells": cells,
                       "schedule": {str(k): v for k, v in sched.items()},
                       "l2": "inputs larger than L2 (46 M cells x 9 x 8 B per RK buffer)",
                       "parallelism": f"boxes sharded over {world} rank(s)"},
            "clocks": clk.summary(),
            "one_at_a_time": {"value": cells * K / (ms_1 * 1e-3), "ms_per_step": ms_1 / K,
                              "gpu_launches": launches_1},
            "gpu_launches": launches_b, "speedup_vs_one_at_a_time": ms_1 / ms_b}
    print(json.dumps(line), flush=True)


def poly_config(n):
    from hormone_b200 import config

    ov = dict(ie=n, je=n, ke=n, mag_on=False, gamma=2.0, gravswitch=3, G=1.0, courant=0.9,
              xi1s=-2.0, xi1e=2.0, xi2s=-2.0, xi2e=2.0, xi3s=-2.0, xi3e=2.0, t_end=1e30, dt_out=1e30)
    for a in (1, 2, 3):
        for tag in ("is", "os", "iv", "ov"):
            ov[f"bc{a}{tag}"] = 3
    return config.resolve("polytrope_cart", overrides=ov)


def run_polytrope(args, rank, world, local_rank):
    """Self-gravitating n=1 polytrope (G=1, K=2/pi, gamma=2) in a 192^3 box
    [-2,2]^3 with hyperbolic gravity, FP64: zone-updates/s over the steps
    (each step = CFL + the gravity sub-cycles + 3 fused RK stages), mass and
    momentum drift over the run, and the L1 error against the oracle on a
    48^3 box of the same set-up."""
    import numpy as np
    import torch

    from hormone_b200 import grid as G, ic
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    n = args.size if args.size != 256 else 192
    cfg = poly_config(n)
    grid = G.make_grid(cfg)
    prims, phi = ic.polytrope_n1(cfg, grid)
    dv = float(grid[0]["dxi"][2] * grid[1]["dxi"][2] * grid[2]["dxi"][2])
    sim = Simulation(cfg, prims, grvphi=phi)
    stream = torch.cuda.ExternalStream(sim.ctx.stream_ptr())
    u0 = sim.state()["u"]
    mass0 = float(u0[0].sum() * dv)
    sim.run(max_steps=args.warmup)
    torch.cuda.synchronize()
    sim.ctx.sync()
    steps = args.poly_steps
    l0 = sim.ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        sim.run(max_steps=steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sim.ctx.launches() - l0
    u1 = sim.state()["u"]
    t_sim = sim.time
    sim.close()
    mass1 = float(u1[0].sum() * dv)
    mom = [float(u1[q].sum() * dv) for q in (1, 2, 3)]
    vdyn = math.sqrt(4.0 / math.pi)  # sqrt(G M / R) of the star
    cells = n ** 3
    value = cells * steps / (ms * 1e-3)
    # L1 against the oracle on a small box, same set-up, step for step
    l1 = None
    cpu = None
    if not args.no_cpu:
        from oracle.oracle import Oracle

        m = 48
        c2 = poly_config(m)
        p2, f2 = ic.polytrope_n1(c2, G.make_grid(c2))
        o = Oracle(c2)
        o.set_prims(p2)
        o.set_gravity_state(f2, None, 0.0)
        o.start()
        s2 = Simulation(c2, p2, grvphi=f2)
        k = 20
        t0 = time.perf_counter()
        for _ in range(k):
            o.step()
        el = time.perf_counter() - t0
        s2.run(max_steps=k)
        a, b = s2.state()["u"], o.u()
        s2.close()
        l1 = {name: float(np.sum(np.abs(a[q] - b[q])) / max(np.sum(np.abs(b[q])), 1e-300))
              for q, name in enumerate(("rho", "m1", "m2", "m3", "E"))}
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": m ** 3 * k / el, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"{m}^3 box of the same set-up, {k} steps ({el:.1f} s) of the CPU restatement, OpenMP"}
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"polytrope-n1-hyperbolic-gravity-{n}^3", "grid": [n, n, n], "box": [-2, 2],
                       "G": 1.0, "K": 2 / math.pi, "gamma": 2.0, "HGfac": cfg["HGfac"], "hgcfl": cfg["hgcfl"],
                       "l2": f"inputs larger than L2 (5 x 8 B x {n}^3 per RK buffer)"},
            "polytrope": {"t": t_sim, "mass_drift": (mass1 - mass0) / mass0,
                          "momentum_drift": math.sqrt(sum(x * x for x in mom)) / (mass0 * vdyn),
                          "l1_vs_oracle_48^3_20_steps": l1},
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


def poly_sph_config(n, xi1s=0.1):
    from hormone_b200 import config

    ov = dict(ie=n[0], je=n[1], ke=n[2], crdnt=2, mag_on=False, gamma=2.0, gravswitch=3, gbtype=1, G=1.0,
              courant=0.9, xi1s=xi1s, xi1e=2.0, t_end=1e30, dt_out=1e30, bc1is=1, bc1iv=1, bc1os=2, bc1ov=2)
    return config.resolve("polytrope_sph", overrides=ov)


def run_polytrope_sph(args, rank, world, local_rank):
    """The n=1 polytrope on a 3-D spherical polar grid (r in [0.1, 2], full
    theta and phi; 160 x 80 x 160 cells) with hyperbolic self-gravity, FP64:
    zone-updates/s over the timed steps (CFL + gravity sub-cycles + 3 fused
    stages), mass drift, and the L1 error against the oracle on a 48 x 24 x 32
    grid of the same set-up over 40 steps."""
    import numpy as np
    import torch

    from hormone_b200 import grid as G, ic
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    n = (160, 80, 160)
    cfg = poly_sph_config(n)
    grid = G.make_grid(cfg)
    prims, phi = ic.polytrope_n1_spherical(cfg, grid)
    dv = G.spherical_dvol(grid, cfg["n"])
    sim = Simulation(cfg, prims, grvphi=phi)
    stream = torch.cuda.ExternalStream(sim.ctx.stream_ptr())
    mass0 = float(np.sum(sim.state()["u"][0] * dv))
    sim.run(max_steps=args.warmup)
    torch.cuda.synchronize()
    sim.ctx.sync()
    steps = args.steps * 20
    l0 = sim.ctx.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        e0.record(stream)
        sim.run(max_steps=steps)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = sim.ctx.launches() - l0
    mass1 = float(np.sum(sim.state()["u"][0] * dv))
    t_sim = sim.time
    sim.close()
    cells = n[0] * n[1] * n[2]
    l1 = cpu = None
    if not args.no_cpu:
        from oracle.oracle import Oracle

        m = (48, 24, 32)
        c2 = poly_sph_config(m)
        p2, f2 = ic.polytrope_n1_spherical(c2, G.make_grid(c2))
        o = Oracle(c2)
        o.set_prims(p2)
        o.set_gravity_state(f2, None, 0.0)
        o.start()
        s2 = Simulation(c2, p2, grvphi=f2)
        k = 40
        t0 = time.perf_counter()
        for _ in range(k):
            o.step()
        el = time.perf_counter() - t0
        s2.run(max_steps=k)
        a, b = s2.state()["u"], o.u()
        s2.close()
        l1 = {name: float(np.sum(np.abs(a[q] - b[q])) / max(np.sum(np.abs(b[q])), 1e-300))
              for q, name in enumerate(("rho", "m1", "m2", "m3", "E"))}
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": m[0] * m[1] * m[2] * k / el, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"{m[0]}x{m[1]}x{m[2]} grid of the same set-up, {k} steps ({el:.1f} s) of the CPU "
                         "restatement, OpenMP"}
    line = {"metric": METRIC, "value": cells * steps / (ms * 1e-3), "unit": METRIC, "n_gpus": 1, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"polytrope-n1-spherical-hyperbolic-gravity-{n[0]}x{n[1]}x{n[2]}",
                       "crdnt": 2, "r": [0.1, 2.0], "G": 1.0, "K": 2 / math.pi, "gamma": 2.0,
                       "HGfac": cfg["HGfac"], "hgcfl": cfg["hgcfl"], "gbtype": 1,
                       "l2": "inputs larger than L2 (5 x 8 B x 2.05 M cells per RK buffer, 8 coefficient planes)"},
            "polytrope": {"t": t_sim, "mass_drift": (mass1 - mass0) / mass0, "l1_vs_oracle_48x24x32_40_steps": l1},
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk.summary()}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_briowu(args, rank=0, world=1, local_rank=0):
    """The Brio-Wu shock tube of the benchmark list (1024 cells on [0,1],
    gamma=2, Bx=0.75, minmod, CFL 0.4, to t=0.1): time to solution of the
    whole run on the device clock (hmn_run), FP64 and mixed, against the
    oracle's CPU run of the same case.  A parity case: ~2000 steps of 1024
    cells are launch-bound on a GPU."""
    import numpy as np
    import torch

    from hormone_b200 import config, grid as G, ic
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    cfg = config.resolve("briowushock_x test", overrides=dict(ie=1024, t_end=100.0, dt_out=100.0, courant=0.4,
                                                              flux_limiter="minmod"))
    prims = ic.make(cfg, G.make_grid(cfg))
    out = {}
    for prec in (0, 1):
        runs = []
        for rep in range(max(1, args.warmup) + 1):
            s = Simulation(cfg, prims, precision=prec)
            stream = torch.cuda.ExternalStream(s.ctx.stream_ptr())
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            s.run_device()
            e1.record(stream)
            e1.synchronize()
            runs.append((e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3, s.tn, s.ctx.launches()))
            st = s.state()
            s.close()
        ms, wall, tn, launches = runs[-1]
        out[prec] = dict(ms=ms, wall_ms=wall, steps=tn, launches=launches, d=st["d"])
    l1 = float(np.sum(np.abs(out[1]["d"] - out[0]["d"])) / np.sum(np.abs(out[0]["d"])))
    cpu = None
    if not args.no_cpu:
        from oracle.oracle import Oracle

        o = Oracle(cfg)
        o.set_prims(prims)
        t0 = time.perf_counter()
        o.start()
        o.run()
        el = time.perf_counter() - t0
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": 1024 * o.scalars()["tn"] / el, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"the whole run ({o.scalars()['tn']} steps, {el:.2f} s) of the CPU restatement"}
    cells = 1024
    r0 = out[0]
    line = {"metric": METRIC, "value": cells * r0["steps"] / (r0["ms"] * 1e-3), "unit": METRIC, "n_gpus": 1,
            "steps": r0["steps"], "warmup": max(1, args.warmup), "ms_per_step": r0["ms"] / r0["steps"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "brio-wu-1024-cells-t0.1", "gamma": 2.0, "limiter": "minmod", "courant": 0.4,
                       "l2": "inputs far smaller than L2 (a launch-bound parity case)"},
            "time_to_solution_ms": {"fp64": r0["ms"], "mixed": out[1]["ms"], "fp64_wall": r0["wall_ms"]},
            "mixed_l1_rho_vs_fp64": l1, "gpu_launches": r0["launches"], "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_sedov(args, rank=0, world=1, local_rank=0):
    """HORMONE's own spherical Sedov-Taylor test (sedov_default: 500 radial
    cells of a spherical polar grid, gamma=1.4, modified MC, to t=0.3):
    time to solution of the whole run on the device clock (hmn_run), FP64
    and mixed, against the oracle's CPU run of the same case.  Launch-bound
    like the Brio-Wu case."""
    import numpy as np
    import torch

    from hormone_b200 import config, grid as G, ic
    from hormone_b200.sim import Simulation

    torch.cuda.set_device(local_rank)
    cfg = config.resolve("sedov_default test")
    prims = ic.make(cfg, G.make_grid(cfg))
    out = {}
    for prec in (0, 1):
        runs = []
        for rep in range(max(1, args.warmup) + 1):
            s = Simulation(cfg, prims, precision=prec)
            stream = torch.cuda.ExternalStream(s.ctx.stream_ptr())
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            s.run_device()
            e1.record(stream)
            e1.synchronize()
            runs.append((e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3, s.tn, s.ctx.launches()))
            d = s.state()["d"]
            s.close()
        out[prec] = runs[-1] + (d,)
    ms, wall, tn, launches, d0 = out[0]
    l1 = float(np.sum(np.abs(out[1][4] - d0)) / np.sum(np.abs(d0)))
    cells = cfg["n"][0]
    cpu = None
    if not args.no_cpu:
        from oracle.oracle import Oracle

        o = Oracle(cfg)
        o.set_prims(prims)
        t0 = time.perf_counter()
        o.start()
        o.run()
        el = time.perf_counter() - t0
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": cells * o.scalars()["tn"] / el, "unit": METRIC, "cores": cores, "kind": "port",
               "sample": f"the whole run ({o.scalars()['tn']} steps, {el:.2f} s) of the CPU restatement"}
    line = {"metric": METRIC, "value": cells * tn / (ms * 1e-3), "unit": METRIC, "n_gpus": 1, "steps": tn,
            "warmup": max(1, args.warmup), "ms_per_step": ms / tn, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "sedov-spherical-500-cells-t0.3", "crdnt": 2, "gamma": 1.4,
                       "limiter": "modified_mc", "l2": "inputs far smaller than L2 (a launch-bound parity case)"},
            "time_to_solution_ms": {"fp64": ms, "mixed": out[1][0], "fp64_wall": wall},
            "mixed_l1_rho_vs_fp64": l1, "gpu_launches": launches, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def run_serve(args, rank=0, world=1, local_rank=0):
    """The serving stream through the continuous-batching server.  With N
    ranks every request goes to one rank (split by cells, in arrival order
    within a rank); latencies are pooled over ranks."""
    from hormone_b200 import serve, shard
    from hormone_b200.batch import Batch

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    reqs = serve.make_requests(args.requests, rate=args.rate, seed=20261203)
    mine = set(shard.my_share([r.cells for r in reqs], rank, world))
    reqs = [r for i, r in enumerate(reqs) if i in mine]
    free, total = torch.cuda.mem_get_info()
    b = Batch(int(free * 0.6), max_sims=1024, precision=args.precision)
    if dist:
        dist.barrier()
    with ClockSampler(local_rank) as clk:
        stats = serve.serve(reqs, b, chunk=8, keep_results=False, policy=args.policy,
                            live_cells=args.live_cells or None)
    b.close()
    if dist:
        allst = [None] * world
        dist.all_gather_object(allst, (stats.latencies, stats.zone_updates, stats.wall_s, stats.completed,
                                       stats.failed, stats.max_live, stats.batch_steps))
        stats.latencies = [x for a in allst for x in a[0]]
        stats.zone_updates = sum(a[1] for a in allst)
        stats.wall_s = max(a[2] for a in allst)
        stats.completed = sum(a[3] for a in allst)
        stats.failed = sum(a[4] for a in allst)
        stats.max_live = max(a[5] for a in allst)
        stats.batch_steps = max(a[6] for a in allst)
    if rank != 0:
        return
    summ = stats.summary()
    line = {"metric": METRIC, "value": summ["zone_updates_per_s"], "unit": METRIC, "n_gpus": world,
            "steps": summ["batch_steps"], "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "mixed", "data": "synthetic",
            "config": {"workload": f"serve-{args.requests}-requests-poisson-{args.rate}/s",
                       "pool_bytes": int(free * 0.6), "parallelism": f"requests sharded over {world} rank(s)",
                       "admission": args.policy, "live_cells_cap": args.live_cells or None},
            "serve": summ, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.workload == "kh-batch":
            run_kh_batch(args, rank, world, local_rank)
        elif args.workload == "serve":
            run_serve(args, rank, world, local_rank)
        elif args.workload == "polytrope-sph":
            run_polytrope_sph(args, rank, world, local_rank)
        elif args.workload == "polytrope":
            run_polytrope(args, rank, world, local_rank)
        elif args.workload == "briowu":
            run_briowu(args, rank, world, local_rank)
        elif args.workload == "sedov":
            run_sedov(args, rank, world, local_rank)
        elif args.decomp == "slab" and world > 1:
            run_slab(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
