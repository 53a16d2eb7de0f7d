"""The error norms of HORMONE's test harness (src/main/tests.f90:46-292).

``compare`` returns the per-variable max, "L1" and L2 norms exactly as
``test`` computes them; a run passes when the largest L2 norm is below
``test_tol`` (tests.f90:168-179).  The scales follow tests.f90:135-157:
velocity components use max(|v|, cs*Mach_tol), field components |B|, the rest
|value|, all floored at machine epsilon, with |v|, |B| and cs taken from the
golden state.
"""
import math

import numpy as np

EPS = np.finfo(np.float64).eps


def _max_norm(var, var0, scale):
    pos = var.max() * var.min()
    if pos > 0.0:
        return float(np.max(np.abs(var / var0 - 1.0)))
    return float(np.max(np.abs(var - var0) / np.maximum(np.abs(var0), scale)))


def _l1_norm(var, var0, scale, w):
    pos = var.max() * var.min()
    if pos > 0.0:
        errsum = np.sum(np.abs(var / var0 - 1.0) * w)
    else:
        errsum = np.sum(np.abs(var - var0) / np.maximum(np.abs(var0), scale) * w)
    return float(math.sqrt(errsum) / math.sqrt(np.sum(w)))


def _window(a, r, fn):
    """fn (max or min filter) over the (2r+1)^3 window clipped at the array
    edges: edge replication adds no value from outside the clipped window."""
    from scipy import ndimage

    return fn(a, size=2 * r + 1, mode="nearest")


_exp = np.frompyfunc(math.exp, 1, 1)


def _l2_norm(var, var0, scale, w, disco_range=3):
    """tests.f90's discontinuity-weighted L2 norm, vectorised: the jump of a
    cell is max(M / max(|q|, floor), |q| / max(m, floor), 1) with M and m the
    largest and smallest |q0| over its clipped neighbourhood (both ratios are
    monotone in the neighbour value, so their maxima are taken at M and m),
    and exp is math.exp cell by cell, so the result equals the cell loop's."""
    from scipy import ndimage

    pos = var.max() * var.min()
    a0 = np.abs(var0)
    big = _window(a0, disco_range, ndimage.maximum_filter)
    small = _window(a0, disco_range, ndimage.minimum_filter)
    if pos <= 0.0:
        base = np.maximum(a0, scale)
        denom = np.maximum(big, scale)
        floor = scale
    else:
        base = var0
        denom = big
        floor = np.zeros_like(var0)
    ay = np.abs(base)
    jump = np.maximum(np.maximum(big / np.maximum(ay, floor), ay / np.maximum(small, floor)), 1.0)
    rel = (var - var0) / denom * _exp(1.0 - jump).astype(np.float64)
    return float(math.sqrt(np.sum(rel ** 2 * w)) / math.sqrt(np.sum(w)))


def compare(sim: dict, gold: dict, cfg: dict, dvol=None, fast_l2_if_identical=True):
    """Norms of ``sim`` against ``gold`` (dicts of (nz,ny,nx) arrays)."""
    labels = ["d", "e", "v1", "v2", "v3"]
    if cfg["mag_on"]:
        labels += ["b1", "b2", "b3"]
        if cfg["dim"] >= 2:
            labels += ["phi"]
    # passive scalars (tests.f90:84-87,106-110): scaled by their own magnitude
    labels += [f"spc{n}" for n in range(cfg.get("nspc", 0))]
    g = gold
    vmag = np.sqrt(g["v1"] ** 2 + g["v2"] ** 2 + g["v3"] ** 2)
    bmag = np.sqrt(g["b1"] ** 2 + g["b2"] ** 2 + g["b3"] ** 2) if cfg["mag_on"] else np.zeros_like(vmag)
    # cs from the golden state (tests.f90:139 calls timestep after readbin)
    gm1 = cfg["gamma"] - 1.0
    vsq = g["v1"] * g["v1"] + g["v2"] * g["v2"] + g["v3"] * g["v3"]
    eint = g["e"] - 0.5 * g["d"] * vsq
    if cfg["mag_on"]:
        eint = eint - 0.5 * (g["b1"] * g["b1"] + g["b2"] * g["b2"] + g["b3"] * g["b3"])
    cs = np.sqrt(cfg["gamma"] * (gm1 * eint) / g["d"])
    w = np.ones_like(vmag) if dvol is None else dvol
    out = {}
    for lab in labels:
        if lab in ("v1", "v2", "v3"):
            scale = np.maximum(vmag, cs * cfg.get("Mach_tol", 1e-5))
        elif lab in ("b1", "b2", "b3"):
            scale = bmag.copy()
        elif lab.startswith("spc"):
            scale = np.abs(g["spc"][int(lab[3:])])
        else:
            scale = np.abs(g[lab])
        scale = np.maximum(scale, EPS)
        ref = g["spc"][int(lab[3:])] if lab.startswith("spc") else g[lab]
        var, var0 = np.asarray(sim[lab], dtype=np.float64), np.asarray(ref, dtype=np.float64)
        same = bool(np.array_equal(var, var0))
        l2 = 0.0 if (same and fast_l2_if_identical) else _l2_norm(var, var0, scale, w)
        out[lab] = dict(max=_max_norm(var, var0, scale), L1=_l1_norm(var, var0, scale, w), L2=l2,
                        identical=same, maxabs=float(np.max(np.abs(var - var0))))
    return out
