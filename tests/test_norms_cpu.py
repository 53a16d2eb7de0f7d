"""The vectorised discontinuity-weighted L2 norm (hormone_b200.norms) equals
the cell-by-cell loop of tests.f90's definition, bit for bit, for fields of
one sign and of both signs, with jumps, on uneven shapes."""
import numpy as np
import pytest

import norms


@pytest.mark.parametrize("shape,signed", [((7, 5, 9), False), ((6, 8, 4), True), ((1, 1, 30), True),
                                          ((3, 11, 1), False)])
def test_l2_norm_vectorised_equals_loop(shape, signed):
    rng = np.random.default_rng(sum(shape))
    var0 = rng.uniform(0.5, 2.0, shape)
    var0[..., : shape[-1] // 2] *= 40.0  # a jump
    if signed:
        var0 = var0 * rng.choice([-1.0, 1.0], shape)
        var0.flat[3] = 0.0
    var = var0 * (1.0 + rng.normal(0.0, 1e-6, shape))
    scale = np.maximum(np.abs(var0), norms.EPS)
    w = rng.uniform(0.5, 1.5, shape)
    a = norms._l2_norm(var, var0, scale, w)
    b = norms._l2_norm_loop(var, var0, scale, w)
    assert a == b, (a, b)
    assert a > 0.0
