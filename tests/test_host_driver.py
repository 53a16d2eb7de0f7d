"""The C ABI from C: tests/host_driver.c, compiled with gcc against
include/hormone_gpu.h, is the host a Fortran ISO_C_BINDING shim stands for.

* The struct layouts the C compiler gives hmn_grid, hmn_params and
  hmn_metric are those of the ctypes mirrors (hormone_b200/capi.py) every
  other test drives the library with, field by field.
* On a GPU, the driver runs HORMONE's step loop (hormone.f90:107-179)
  through the C entry points on the Brio-Wu golden set-up and reproduces the
  reference's golden dump (tests/golden/briowushock_x.npz) bit for bit."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from hormone_b200 import capi, grid as G, ic

import cases

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "host_driver.c")
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "hormone_b200")


def _gcc():
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    return cc


def test_struct_layouts_match_the_ctypes_mirrors(tmp_path):
    exe = str(tmp_path / "host_driver_layout")
    subprocess.run([_gcc(), "-std=c99", "-Wall", "-Werror", "-DHMN_LAYOUT_ONLY", "-I", INC, SRC, "-o", exe],
                   check=True)
    out = subprocess.run([exe, "layout"], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        key, val = line.rsplit(" ", 1)
        got[key] = int(val)
    for name, cls in (("hmn_grid", capi.HmnGrid), ("hmn_params", capi.HmnParams), ("hmn_metric", capi.HmnMetric)):
        assert got[f"sizeof {name}"] == ctypes.sizeof(cls), name
        for field, _ in cls._fields_:
            assert got[f"{name}.{field}"] == getattr(cls, field).offset, (name, field)
        assert len([k for k in got if k.startswith(name + ".")]) == len(cls._fields_), name


def _write_input(path, cfg, prims):
    grid = G.make_grid(cfg)
    st = ic.to_state(cfg, prims)
    glm = int(bool(cfg["mag_on"]) and cfg["dim"] > 1)
    with open(path, "wb") as f:
        np.asarray(cfg["n"], dtype="<i4").tofile(f)
        np.asarray(cfg["bc"], dtype="<i4").reshape(-1).tofile(f)
        np.asarray([cfg["rktype"], cfg["grktype"], cfg["limiter_code"], int(cfg["mag_on"]), cfg["gravswitch"],
                    cfg["maxtngrv"], cfg["outstyle"], cfg["endstyle"], st["u"].shape[0], glm], dtype="<i4").tofile(f)
        np.asarray([cfg["gamma"], cfg["courant"], cfg["alpha9wave"], cfg["HGfac"], cfg["hgcfl"], cfg["alphagrv"],
                    cfg["G"], cfg["t_out"], cfg["dt_out"], cfg["t_end"]], dtype="<f8").tofile(f)
        for a in range(3):
            for key in ("x", "xi", "dx", "dxi", "idx", "idxi"):
                arr = np.ascontiguousarray(grid[a][key], dtype="<f8")
                assert arr.size == cfg["n"][a] + 4
                arr.tofile(f)
        np.ascontiguousarray(st["u"], dtype="<f8").tofile(f)
        for p in st["prim"]:
            np.ascontiguousarray(p, dtype="<f8").tofile(f)
    return st["u"].shape


@pytest.mark.gpu
def test_c_host_loop_reproduces_the_golden_dump(tmp_path):
    if not os.path.exists(capi.LIB_PATH):
        pytest.fail("libhormone_b200.so is missing")
    exe = str(tmp_path / "host_driver")
    subprocess.run([_gcc(), "-std=c99", "-Wall", "-Werror", "-I", INC, SRC, "-L", LIBDIR, "-lhormone_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    name = "briowushock_x"
    cfg, prims = cases.golden_case(name)
    inp, outp = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    ushape = _write_input(inp, cfg, prims)
    subprocess.run([exe, "run", inp, outp], check=True)
    raw = open(outp, "rb").read()
    tn = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    t = float(np.frombuffer(raw[4:12], dtype="<f8")[0])
    vals = np.frombuffer(raw[12:], dtype="<f8")
    cells = int(np.prod(cfg["n"]))
    nvar = ushape[0]
    assert vals.size == (nvar + 9) * cells
    shape = (cfg["n"][2], cfg["n"][1], cfg["n"][0])
    prim = {k: vals[(nvar + q) * cells:(nvar + q + 1) * cells].reshape(shape)
            for q, k in enumerate(("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi"))}
    gold = dict(np.load(os.path.join(HERE, "golden", name + ".npz")))
    assert tn == int(gold["tn"]) and t == float(gold["time"])
    for k in ("d", "e", "v1", "v2", "v3", "b1", "b2", "b3"):
        if k in gold:
            assert np.array_equal(prim[k], gold[k]), k
