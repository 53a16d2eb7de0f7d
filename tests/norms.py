"""The error norms of HORMONE's test harness (hormone_b200.norms), plus the
cell-by-cell loop of the discontinuity-weighted L2 norm that the vectorised
one is checked against."""
import math

import numpy as np

from hormone_b200.norms import EPS, _l1_norm, _l2_norm, _max_norm, compare  # noqa: F401


def _l2_norm_loop(var, var0, scale, w, disco_range=3):
    pos = var.max() * var.min()
    nz, ny, nx = var.shape
    rel = np.zeros_like(var)
    for k in range(nz):
        kl, ku = min(disco_range, k), min(disco_range, nz - 1 - k)
        for j in range(ny):
            jl, ju = min(disco_range, j), min(disco_range, ny - 1 - j)
            for i in range(nx):
                il, iu = min(disco_range, i), min(disco_range, nx - 1 - i)
                nb = var0[k - kl:k + ku + 1, j - jl:j + ju + 1, i - il:i + iu + 1]
                base = var0[k, j, i]
                denom = np.max(np.abs(nb))
                floor = 0.0
                if pos <= 0.0:
                    base = max(abs(base), scale[k, j, i])
                    denom = max(denom, scale[k, j, i])
                    floor = scale[k, j, i]
                ax = np.abs(nb)
                ay = abs(base)
                ratio = np.maximum(np.maximum(ax / max(ay, floor), ay / np.maximum(ax, floor)), 1.0)
                jump = np.max(ratio)
                rel[k, j, i] = (var[k, j, i] - var0[k, j, i]) / denom * math.exp(1.0 - jump)
    return float(math.sqrt(np.sum(rel ** 2 * w)) / math.sqrt(np.sum(w)))


