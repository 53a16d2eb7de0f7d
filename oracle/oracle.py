"""ctypes binding of the CPU oracle (hormone_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / ``--impl reference`` legs as the checker.  The
product package ``hormone_b200`` never imports this module.

The oracle is a pass-by-pass C restatement of HORMONE's FP64 explicit step
(src/main/hydro.f90:15-52 and the routines it calls); see the header of
hormone_oracle.c for the file:line map.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)

# accessor codes of hmo_get
FIELDS = {"d": 0, "p": 1, "e": 2, "v1": 3, "v2": 4, "v3": 5, "b1": 6, "b2": 7, "b3": 8, "phi": 9,
          "eint": 10, "cs": 11, "grvphi": 12, "grvpsi": 13}


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        L.hmo_create.restype = _P
        L.hmo_create.argtypes = [_I, _I, _I, _I, _I, _I, _D, _D, _D, ctypes.POINTER(_I)]
        L.hmo_destroy.argtypes = [_P]
        L.hmo_set_times.argtypes = [_P, _D, _D, _D, _I, _I, _I]
        L.hmo_set_test_mode.argtypes = [_P]
        L.hmo_set_gravity.argtypes = [_P, _I, _D, _D, _D, _D, _I, _I]
        L.hmo_make_uniform_axis.argtypes = [_P, _I, _D, _D]
        L.hmo_make_axis.argtypes = [_P, _I, _D, _DP]
        L.hmo_make_geometric_axis.argtypes = [_P, _I, _D, _D, _D]
        L.hmo_make_geometric_axis.restype = _I
        L.hmo_make_spherical.argtypes = [_P, _I, _D, _D, _D, _I]
        L.hmo_make_spherical.restype = _I
        L.hmo_make_cylindrical.argtypes = [_P, _I, _D, _D, _D, _I, _D, _D, _D]
        L.hmo_make_cylindrical.restype = _I
        L.hmo_get_metric.argtypes = [_P, _I, _DP]
        L.hmo_get_metric.restype = _I
        L.hmo_get_axis.argtypes = [_P, _I] + [_DP] * 6
        L.hmo_set_prims.argtypes = [_P] + [_DP] * 9
        L.hmo_set_grvphi.argtypes = [_P, _DP, _DP]
        L.hmo_set_species.argtypes = [_P, _I]
        L.hmo_set_species.restype = _I
        L.hmo_set_spc.argtypes = [_P, _I, _DP]
        L.hmo_set_dirichlet.argtypes = [_P, _I, _I, _DP]
        L.hmo_set_dirichlet.restype = _I
        L.hmo_set_flux_boundary.argtypes = [_P, _DP]
        L.hmo_set_flux_boundary.restype = _I
        L.hmo_gravity_setup.argtypes = [_P, _D]
        L.hmo_start.argtypes = [_P]
        L.hmo_start.restype = _I
        L.hmo_step.argtypes = [_P]
        L.hmo_step.restype = _I
        L.hmo_run.argtypes = [_P, _I]
        L.hmo_run.restype = _I
        L.hmo_timestep.argtypes = [_P]
        L.hmo_timestep.restype = _I
        L.hmo_hydro_step.argtypes = [_P]
        L.hmo_hydro_step.restype = _I
        L.hmo_gravity.argtypes = [_P]
        L.hmo_gravity.restype = _I
        L.hmo_phidamp.argtypes = [_P]
        L.hmo_get.argtypes = [_P, _I, _DP]
        L.hmo_get.restype = _I
        L.hmo_scalars.argtypes = [_P, _DP]
        L.hmo_set_scalars.argtypes = [_P, _D, _I, _D, _D]
        L.hmo_error.argtypes = [_P, ctypes.POINTER(_I)]
        L.hmo_nvar.argtypes = [_P]
        L.hmo_nvar.restype = _I
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    return a.ctypes.data_as(_DP)


class Oracle:
    """One simulation advanced by the CPU restatement.

    ``cfg`` is a resolved configuration dict from ``hormone_b200.config``
    (the keys used here mirror HORMONE's namelist names).
    """

    def __init__(self, cfg: dict):
        L = lib()
        self.cfg = cfg
        n = cfg["n"]
        self.shape = (n[2], n[1], n[0])  # k, j, i  (C order, x fastest)
        bc = (ctypes.c_int * 12)(*[int(v) for v in np.asarray(cfg["bc"], dtype=np.int64).reshape(-1)])
        self.h = L.hmo_create(n[0], n[1], n[2], int(cfg["mag_on"]), int(cfg["limiter_code"]), int(cfg["rktype"]),
                              float(cfg["gamma"]), float(cfg["courant"]), float(cfg["alpha9wave"]), bc)
        if cfg.get("gravswitch", 0):
            L.hmo_set_gravity(self.h, int(cfg["gravswitch"]), float(cfg["HGfac"]), float(cfg["hgcfl"]),
                              float(cfg["alphagrv"]), float(cfg["G"]), int(cfg["grktype"]), int(cfg["maxtngrv"]))
        mesh_keys = ("imesh", "jmesh", "kmesh")
        if int(cfg.get("crdnt", 0)) == 2:
            imesh = int(cfg.get("imesh", 0)) if n[0] > 1 else 0
            lo, hi = cfg["extent"][0]
            if L.hmo_make_spherical(self.h, imesh, float(lo), float(hi), float(cfg.get("x1min", 0.0)),
                                    int(bool(cfg.get("eq_sym", False)))) != 0:
                raise ValueError("spherical grid: bad settings")
        if int(cfg.get("crdnt", 0)) == 1:
            (r0, r1), (z0, z1) = cfg["extent"][0], cfg["extent"][2]
            if L.hmo_make_cylindrical(self.h, int(cfg.get("imesh", 0)) if n[0] > 1 else 0, float(r0), float(r1),
                                      float(cfg.get("x1min", 0.0)), int(cfg.get("kmesh", 0)) if n[2] > 1 else 0,
                                      float(z0), float(z1), float(cfg.get("x3min", 0.0))) != 0:
                raise ValueError("cylindrical grid: bad settings")
        for a, (lo, hi) in enumerate(cfg["extent"]):
            if int(cfg.get("crdnt", 0)) in (1, 2):
                break
            if cfg["n"][a] > 1 and int(cfg.get(mesh_keys[a], 0)) == 1:
                xmin = float(cfg[("x1min", "x2min", "x3min")[a]])
                if L.hmo_make_geometric_axis(self.h, a, float(lo), float(hi), xmin) != 0:
                    raise ValueError("geometrical series mesh: bad xmin")
            else:
                L.hmo_make_uniform_axis(self.h, a, float(lo), float(hi))
        L.hmo_set_times(self.h, 0.0, float(cfg["t_end"]), float(cfg["dt_out"]), int(cfg["outstyle"]),
                        int(cfg["endstyle"]), int(cfg["tnlim"]))
        if cfg.get("is_test", False):
            L.hmo_set_test_mode(self.h)
        self.nspc = int(cfg.get("nspc", 0))
        if self.nspc:
            L.hmo_set_species(self.h, self.nspc)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().hmo_destroy(h)
            self.h = None

    # -- set-up ---------------------------------------------------------
    def axis(self, a):
        n = self.cfg["n"][a] + 4
        arrs = [np.zeros(n) for _ in range(6)]
        lib().hmo_get_axis(self.h, a, *[_dp(x) for x in arrs])
        return dict(zip(["x", "xi", "dx", "dxi", "idx", "idxi"], arrs))

    def metric(self) -> dict:
        """Spherical metric factors: detg1, idetg1, sx1 (n0+4) and sini,
        cosi, scot, sinc, sisin (n1+4)."""
        out = {}
        for w, name in enumerate(("detg1", "idetg1", "sx1", "sini", "cosi", "scot", "sinc", "sisin")):
            a = np.zeros(self.cfg["n"][0 if w < 3 else 1] + 4)
            lib().hmo_get_metric(self.h, w, _dp(a))
            out[name] = a
        return out

    def set_prims(self, prims: dict):
        f = {k: (np.ascontiguousarray(prims[k], dtype=np.float64).reshape(-1) if prims.get(k) is not None else None)
             for k in ["d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi"]}
        self._keep = f
        if self.nspc:
            spc = np.ascontiguousarray(prims["spc"], dtype=np.float64)
            self._keep_spc = spc
            for n in range(self.nspc):
                lib().hmo_set_spc(self.h, n, _dp(spc[n].reshape(-1)))
        lib().hmo_set_prims(self.h, *[_dp(f[k]) for k in ["d", "p", "v1", "v2", "v3", "b1", "b2", "b3", "phi"]])

    def set_dirichlet(self, axis: int, side: int, vals):
        """Ghost values of a code-9 face, laid out as for hmn_set_dirichlet."""
        a = np.ascontiguousarray(vals, dtype=np.float64)
        self._keep_dir = getattr(self, "_keep_dir", {})
        self._keep_dir[(axis, side)] = a
        lib().hmo_set_dirichlet(self.h, int(axis), int(side), _dp(a.reshape(-1)))

    def set_flux_boundary(self, flux):
        """Boundary code 10: the inner x3 face's flux (9 + nspc values)."""
        a = np.ascontiguousarray(flux, dtype=np.float64)
        self._keep_fb = a
        lib().hmo_set_flux_boundary(self.h, _dp(a))

    def set_gravity_state(self, grvphi, grvpsi=None, cgrav_old=0.0):
        a = np.ascontiguousarray(grvphi, dtype=np.float64).reshape(-1)
        b = None if grvpsi is None else np.ascontiguousarray(grvpsi, dtype=np.float64).reshape(-1)
        self._keepg = (a, b)
        lib().hmo_set_grvphi(self.h, _dp(a), _dp(b))
        lib().hmo_gravity_setup(self.h, float(cgrav_old))

    # -- stepping -------------------------------------------------------
    def start(self):
        self._check(lib().hmo_start(self.h))

    def step(self) -> bool:
        rc = lib().hmo_step(self.h)
        self._check(rc)
        return rc == 1

    def run(self, max_steps=10 ** 9) -> bool:
        rc = lib().hmo_run(self.h, int(max_steps))
        self._check(rc)
        return rc == 1

    def timestep(self):
        self._check(lib().hmo_timestep(self.h))

    def hydro_step(self):
        self._check(lib().hmo_hydro_step(self.h))

    def gravity(self):
        self._check(lib().hmo_gravity(self.h))

    def phidamp(self):
        lib().hmo_phidamp(self.h)

    def _check(self, rc):
        if rc < 0:
            e = (ctypes.c_int * 4)()
            lib().hmo_error(self.h, e)
            raise RuntimeError(f"oracle error {e[0]} at cell ({e[1]},{e[2]},{e[3]})")

    # -- state ------------------------------------------------------------
    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.shape)
        if name in FIELDS:
            code = FIELDS[name]
        elif name.startswith("spc"):
            code = 30 + int(name[3:])  # 'spc0', 'spc1', ...
        else:
            code = 20 + int(name[1:])  # 'u0'..'u8'
        if lib().hmo_get(self.h, code, _dp(out)) != 0:
            raise KeyError(name)
        return out

    def u(self) -> np.ndarray:
        nv = lib().hmo_nvar(self.h)
        return np.stack([self.get(f"u{q}") for q in range(nv)])

    def scalars(self) -> dict:
        s = np.zeros(11)
        lib().hmo_scalars(self.h, _dp(s))
        keys = ["time", "dt", "ch", "cfmax", "cgrav", "dtgrav", "dtg_unit", "grvtime", "cgrav_old", "tn", "t_out"]
        out = dict(zip(keys, s.tolist()))
        out["tn"] = int(out["tn"])
        return out

    def set_scalars(self, time, tn, grvtime=0.0, cgrav_old=0.0):
        lib().hmo_set_scalars(self.h, float(time), int(tn), float(grvtime), float(cgrav_old))
