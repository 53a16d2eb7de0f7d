"""The Fortran host's layout: module arrays with two ghost layers per side
(u(is-2:ie+2,js-2:je+2,ks-2:ke+2,1:ufnmax), d(is-2:ie+2,...), spc(1:spn,...)).
A context created with ghost = 2 reads and writes only the interior of such
arrays and gives bit for bit the packed-layout run."""
import numpy as np
import pytest

from hormone_b200 import capi, grid as G, ic

import cases

pytestmark = pytest.mark.gpu
PRIM = ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")


def _pad(a, g=2, fill=np.nan):
    out = np.full(tuple(s + 2 * g for s in a.shape[-3:]), fill) if a.ndim == 3 else \
        np.full(a.shape[:-3] + tuple(s + 2 * g for s in a.shape[-3:]), fill)
    out[..., g:-g, g:-g, g:-g] = a
    return out


def _run(ctx, cfg, steps):
    t = 0.0
    for _ in range(steps):
        dt, ch = ctx.timestep(t, cfg["t_out"], cfg["t_end"])
        ctx.hydro_step()
        if cfg["mag_on"] and cfg["dim"] > 1:
            ctx.phidamp()
        t = t + dt
    return t


@pytest.mark.parametrize("make", [lambda: cases.ot3d(12), lambda: cases.riemann3d(nspc=2)])
def test_ghosted_host_arrays_match_packed(make):
    cfg, prims = make()
    grid = G.make_grid(cfg)
    st = ic.to_state(cfg, prims)
    packed = capi.Context(cfg, grid)
    packed.upload(u=st["u"], prim=list(st["prim"]))
    ghosted = capi.Context(cfg, grid, ghost=2)
    ghosted.upload(u=_pad(st["u"]), prim=[_pad(p) for p in st["prim"]])
    if cfg.get("nspc", 0):
        packed.upload_scalars(st["spc"])
        # species fastest with ghosts: spc(1:spn, i, j, k)
        spc = np.moveaxis(_pad(st["spc"]), 0, -1)
        lib = capi.lib()
        a = np.ascontiguousarray(spc)
        assert lib.hmn_upload_scalars(ghosted.h, capi._dp(a)) == 0
    assert _run(packed, cfg, 4) == _run(ghosted, cfg, 4)
    a, b = packed.download(), ghosted.download()
    for k in a:
        inner = b[k][..., 2:-2, 2:-2, 2:-2]
        assert np.array_equal(a[k], inner), k
        # the ghost layers of the host arrays are not written (they keep the NaN fill)
        shell = b[k].copy()
        shell[..., 2:-2, 2:-2, 2:-2] = np.nan
        assert np.isnan(shell).all(), k
    if cfg.get("nspc", 0):
        out = np.full(a["d"].shape[:0] + tuple(s + 4 for s in a["d"].shape) + (cfg["nspc"],), np.nan)
        assert capi.lib().hmn_download_scalars(ghosted.h, capi._dp(out)) == 0
        got = np.moveaxis(out[2:-2, 2:-2, 2:-2, :], -1, 0)
        assert np.array_equal(got, packed.download_scalars())
    packed.close()
    ghosted.close()
