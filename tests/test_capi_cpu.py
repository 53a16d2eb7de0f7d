"""CPU-side checks of the boundary: the library loads without a GPU and
exports every entry point include/hormone_gpu.h declares; host logic
(namelists, grid, dump format) behaves as the reference's."""
import os

import numpy as np
import pytest

from hormone_b200 import binio, capi, config, grid as G


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = capi.header_functions()
    assert "hmn_hydro_step" in names and "hmn_timestep" in names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_namelist_parser_reads_fortran_syntax():
    txt = """! comment
&gridcon  xi1s=0d0 xi1e=1d0 is=1 ie=500 js=1 je=1 fmr_lvl(1:20)=0 /
&eos_con eostype = 0 gamma=1.6666666666666667d0 /
&simucon crdnt=0 mag_on=.true. flux_limiter='minmod' courant=4d-1 /"""
    g = config.parse_namelists(txt)
    assert g["gridcon"]["ie"] == 500 and g["gridcon"]["xi1e"] == 1.0
    assert g["eos_con"]["gamma"] == 1.6666666666666667
    assert g["simucon"]["mag_on"] is True and g["simucon"]["flux_limiter"] == "minmod"
    assert g["simucon"]["courant"] == 0.4


def test_parameter_file_layers(tmp_path):
    pf = tmp_path / "parameters"
    pf.write_text("&simucon courant=0.5d0 flux_limiter='minmod' /\n&gridcon ie=64 /\n")
    cfg = config.resolve("sodshock_x", parafile=str(pf))
    assert cfg["courant"] == 0.5 and cfg["limiter_code"] == 1 and cfg["n"] == [64, 1, 1]
    # " test" ignores the user file (setup.f90:44-56) and sets t_out = t_end
    cfg = config.resolve("sodshock_x test", parafile=str(pf))
    assert cfg["courant"] == 0.9 and cfg["n"] == [500, 1, 1] and cfg["t_out"] == cfg["t_end"] == 200 * 1e-3


def test_checksetup_boundary_defaults_and_errors():
    cfg = config.resolve("briowushock_y test")
    assert cfg["bc"][0].tolist() == [[2, 2], [2, 2]] and cfg["bc"][2].tolist() == [[3, 3], [3, 3]]
    assert cfg["nvar"] == 8 and not cfg["glm"]
    assert config.resolve("orszagtang_xy test")["nvar"] == 9
    with pytest.raises(ValueError):
        config.resolve("sodshock_x", overrides=dict(bc1is=0, bc1os=3))  # periodic on one side only
    with pytest.raises(ValueError):
        config.resolve("sodshock_x", overrides=dict(courant=1.5))


def test_grid_matches_gridset_running_sums():
    ax = G.uniform_axis(500, 0.0, 1.0)
    assert ax["x"][2] == 0.001 and ax["xi"][1] == 0.0
    # centres are running sums, not xis+(i+1/2)h
    x = [ax["x"][1]]
    for i in range(2, 504):
        x.append(x[-1] + ax["dx"][i])
    assert np.array_equal(np.array(x), ax["x"][1:])


def test_bin_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    f = {k: rng.standard_normal((3, 4, 5)) for k in ("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")}
    path = str(tmp_path / "bin00001s.dat")
    binio.writebin(path, 17, 0.25, f, mag_on=True)
    back = binio.readbin(path, (5, 4, 3), mag_on=True)
    assert back["tn"] == 17 and back["time"] == 0.25
    for k, v in f.items():
        assert np.array_equal(back[k], v)


def test_golden_fixture_format_matches_reference_dump():
    root = os.environ.get("HORMONE_REF")
    ref = os.path.join(root, "tests", "briowushock_x.bin") if root else None
    if ref is None or not os.path.exists(ref):
        pytest.skip("reference tree not given (HORMONE_REF)")
    cfg = config.resolve("briowushock_x test")
    data = binio.readbin(ref, cfg["n"], cfg["mag_on"])
    again = binio.writebin(None, data["tn"], data["time"], data, mag_on=True)
    assert again == open(ref, "rb").read()


def test_geometric_mesh_matches_the_oracle_restatement():
    """imesh=1 (utils.f90:351-404): the host grid and the oracle's C
    restatement build the same arrays, and the widths grow by one ratio."""
    import numpy as np

    from hormone_b200 import config, grid as G
    from oracle.oracle import Oracle

    cfg = config.resolve("riemann", overrides=dict(ie=40, je=24, ke=1, imesh=1, x1min=0.01, jmesh=1, x2min=0.03,
                                                    xi1s=0.0, xi1e=1.0, xi2s=-0.5, xi2e=0.5))
    grid = G.make_grid(cfg)
    o = Oracle(cfg)
    for a in range(2):
        ax = o.axis(a)
        for k in G.AXIS_KEYS:
            assert np.array_equal(ax[k], grid[a][k]), (a, k)
    w = grid[0]["dxi"][2:-2]
    r = w[1:] / w[:-1]
    assert w[0] == 0.01 and np.allclose(r, r[0]) and r[0] > 1.0
    assert abs(grid[0]["xi"][-3] - 1.0) < 1e-9  # the last face lands on xi1e


@pytest.mark.parametrize("n,imesh,xi1s,grav", [((500, 1, 1), 0, 0.0, 0), ((24, 16, 1), 0, 0.0, 0),
                                               ((16, 12, 8), 0, 0.0, 0), ((20, 1, 8), 1, 0.1, 0),
                                               ((10, 5, 4), 0, 0.2, 0), ((20, 16, 1), 1, 0.1, 3),
                                               ((16, 8, 8), 0, 0.2, 3)])
def test_spherical_grid_matches_the_oracle_restatement(n, imesh, xi1s, grav):
    """crdnt=2 (gridset.f90:294-423, metric.f90:102-151): the host's axes,
    volumetric centres, quad-precision sin/cos and metric factors equal the
    oracle's C restatement (which uses libquadmath) bit for bit."""
    import numpy as np

    from hormone_b200 import config, grid as G
    from oracle.oracle import Oracle

    cfg = config.resolve("spherical", overrides=dict(ie=n[0], je=n[1], ke=n[2], crdnt=2, xi1s=xi1s, xi1e=1.0,
                                                      imesh=imesh, x1min=0.03, gravswitch=grav, gbtype=1))
    assert cfg["bc"][1].tolist() == ([[1, 1], [1, 1]] if n[1] > 1 else [[3, 3], [3, 3]])
    grid = G.make_grid(cfg)
    o = Oracle(cfg)
    for a in range(3):
        ax = o.axis(a)
        for k in G.AXIS_KEYS:
            assert np.array_equal(ax[k], grid[a][k]), (a, k)
    m = o.metric()
    for name, a, key in (("detg1", 0, "detg"), ("idetg1", 0, "idetg"), ("sx1", 0, "sx"),
                         ("sini", 1, "sini"), ("cosi", 1, "cosi"), ("scot", 1, "scot"),
                         ("sinc", 1, "sinc"), ("sisin", 1, "sisin")):
        assert np.array_equal(m[name], grid[a][key]), name
    dv = G.spherical_dvol(grid, cfg["n"])
    full = 4.0 / 3.0 * np.pi * (1.0 - xi1s ** 3)
    assert abs(dv.sum() / full - 1.0) < 1e-12  # the cells tile the spherical shell


@pytest.mark.parametrize("n,imesh,kmesh,xi1s", [((40, 1, 32), 0, 0, 0.0), ((30, 1, 1), 1, 0, 0.0),
                                               ((24, 1, 20), 1, 1, 0.1)])
def test_cylindrical_grid_matches_the_oracle_restatement(n, imesh, kmesh, xi1s):
    """crdnt=1 (gridset.f90:145-292, metric.f90:53-100): the host's axes,
    volumetric R centres and metric factors equal the oracle's bit for bit;
    a solved phi axis is refused."""
    import numpy as np

    from hormone_b200 import config, grid as G
    from oracle.oracle import Oracle

    cfg = config.resolve("cyl", overrides=dict(ie=n[0], je=n[1], ke=n[2], crdnt=1, xi1s=xi1s, xi1e=1.0, xi3s=-0.5,
                                                xi3e=0.5, imesh=imesh, x1min=0.03, kmesh=kmesh, x3min=0.04))
    grid = G.make_grid(cfg)
    o = Oracle(cfg)
    for a in range(3):
        ax = o.axis(a)
        for k in G.AXIS_KEYS:
            assert np.array_equal(ax[k], grid[a][k]), (a, k)
    m = o.metric()
    for name, key in (("detg1", "detg"), ("idetg1", "idetg"), ("sx1", "sx")):
        assert np.array_equal(m[name], grid[0][key]), name
    with pytest.raises(ValueError):
        config.resolve("cyl", overrides=dict(ie=8, je=8, ke=8, crdnt=1))
