"""ctypes binding of libhormone_b200.so (the C ABI of include/hormone_gpu.h).

This is the Python side of the same boundary a Fortran ISO_C_BINDING shim
binds (the shim keeps the reference's timestep, gravity, hydro_step and
phidamp names around these entry points).  There is no CPU fallback: if the library or a
CUDA device is missing, creating a context raises.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhormone_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "hormone_gpu.h")

HMN_OK, HMN_EINVAL, HMN_ENEG_EINT, HMN_ECUDA, HMN_EBADCFG, HMN_ENOMEM, HMN_ETIMEOUT = 0, -1, -2, -3, -4, -5, -6
ERRORS = {HMN_EINVAL: "HMN_EINVAL", HMN_ENEG_EINT: "HMN_ENEG_EINT", HMN_ECUDA: "HMN_ECUDA",
          HMN_EBADCFG: "HMN_EBADCFG", HMN_ENOMEM: "HMN_ENOMEM", HMN_ETIMEOUT: "HMN_ETIMEOUT"}

_D, _I, _P = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
_DPP = ctypes.POINTER(_DP)


class HmnGrid(ctypes.Structure):
    _fields_ = [("n", _I * 3), ("ghost", _I), ("bc", _I * 12),
                ("x", _DP * 3), ("xi", _DP * 3), ("dx", _DP * 3), ("dxi", _DP * 3), ("idx", _DP * 3),
                ("idxi", _DP * 3)]


class HmnParams(ctypes.Structure):
    _fields_ = [("gamma", _D), ("courant", _D), ("alpha9wave", _D), ("HGfac", _D), ("hgcfl", _D),
                ("alphagrv", _D), ("G", _D), ("rktype", _I), ("grktype", _I), ("limiter", _I), ("mag_on", _I),
                ("gravswitch", _I), ("maxtngrv", _I), ("outstyle", _I), ("endstyle", _I), ("precision", _I),
                ("nspc", _I)]


class HmnMetric(ctypes.Structure):
    _fields_ = [(k, _DP) for k in ("detg1", "idetg1", "sx1", "sini", "cosi", "scot", "sinc", "sisin")]


class HmnError(RuntimeError):
    def __init__(self, code, where="", cell=None):
        self.code = code
        self.cell = cell
        msg = f"{ERRORS.get(code, code)} in {where}"
        if cell is not None:
            msg += f" at cell {cell}"
        super().__init__(msg)


_lib = None


def header_functions():
    """Names of the functions declared in include/hormone_gpu.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(hmn_\w+)\s*\(", txt)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m hormone_b200.build` "
                               "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.hmn_create.argtypes = [ctypes.POINTER(HmnGrid), ctypes.POINTER(HmnParams), ctypes.POINTER(_P)]
        L.hmn_upload.argtypes = [_P, _DP, _DPP, _DP, _DP]
        L.hmn_timestep.argtypes = [_P, _D, _D, _D, _DP, _DP]
        L.hmn_gravity_step.argtypes = [_P, _D, _D, _I]
        L.hmn_hydro_step.argtypes = [_P]
        L.hmn_phidamp.argtypes = [_P]
        L.hmn_download.argtypes = [_P, _DP, _DPP, _DP, _DP]
        L.hmn_download_pressure.argtypes = [_P, _DP]
        L.hmn_run.argtypes = [_P, _DP, _D, _I, ctypes.POINTER(_I)]
        L.hmn_last_error.argtypes = [_P] + [ctypes.POINTER(_I)] * 5
        L.hmn_launch_count.argtypes = [_P]
        L.hmn_launch_count.restype = ctypes.c_longlong
        L.hmn_sync.argtypes = [_P]
        L.hmn_evo.argtypes = [_P, _DP]
        L.hmn_destroy.argtypes = [_P]
        L.hmn_set_gravity_clock.argtypes = [_P, _D, _D]
        L.hmn_gravity_clock.argtypes = [_P, _DP, _DP]
        L.hmn_checkpoint_begin.argtypes = [_P, _DP, _DPP, _DP, _DP, _DP]
        L.hmn_upload_scalars.argtypes = [_P, _DP]
        L.hmn_set_dirichlet.argtypes = [_P, _I, _I, _DP]
        L.hmn_set_metric.argtypes = [_P, _I, ctypes.POINTER(HmnMetric)]
        L.hmn_set_flux_boundary.argtypes = [_P, _I, _I, _DP]
        L.hmn_download_scalars.argtypes = [_P, _DP]
        L.hmn_checkpoint_wait.argtypes = [_P]
        L.hmn_stream.argtypes = [_P]
        L.hmn_stream.restype = _P
        L.hmn_timestep_noalloc.argtypes = [ctypes.POINTER(HmnGrid), ctypes.POINTER(HmnParams), _P, _D, _D, _D, _P, _P]
        L.hmn_timestep_noalloc.restype = _I
        for name in ("hmn_create", "hmn_upload", "hmn_timestep", "hmn_gravity_step", "hmn_hydro_step", "hmn_phidamp",
                     "hmn_download", "hmn_download_pressure", "hmn_run", "hmn_last_error", "hmn_sync", "hmn_destroy",
                     "hmn_set_gravity_clock", "hmn_gravity_clock", "hmn_checkpoint_begin", "hmn_checkpoint_wait",
                     "hmn_upload_scalars", "hmn_download_scalars", "hmn_set_dirichlet", "hmn_set_metric",
                     "hmn_set_flux_boundary", "hmn_evo"):
            getattr(L, name).restype = _I
        _lib = L
    return _lib


def _dp(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_DP)


def grid_struct(cfg: dict, grid):
    """hmn_grid for a resolved configuration; returns (struct, arrays to keep alive)."""
    keep = []
    g = HmnGrid()
    for a in range(3):
        g.n[a] = cfg["n"][a]
    g.ghost = 0
    bc = np.asarray(cfg["bc"], dtype=np.int32).reshape(-1)
    for q in range(12):
        g.bc[q] = int(bc[q])
    for key in ("x", "xi", "dx", "dxi", "idx", "idxi"):
        arr = getattr(g, key)
        for a in range(3):
            v = np.ascontiguousarray(grid[a][key], dtype=np.float64)
            keep.append(v)
            arr[a] = _dp(v)
    return g, keep


def params_struct(cfg: dict, precision: int = 0) -> HmnParams:
    return HmnParams(gamma=cfg["gamma"], courant=cfg["courant"], alpha9wave=cfg["alpha9wave"], HGfac=cfg["HGfac"],
                     hgcfl=cfg["hgcfl"], alphagrv=cfg["alphagrv"], G=cfg["G"], rktype=cfg["rktype"],
                     grktype=cfg["grktype"], limiter=cfg["limiter_code"], mag_on=int(cfg["mag_on"]),
                     gravswitch=cfg["gravswitch"], maxtngrv=cfg["maxtngrv"], outstyle=cfg["outstyle"],
                     endstyle=cfg["endstyle"], precision=precision, nspc=int(cfg.get("nspc", 0)))


class Context:
    """One simulation resident on the GPU (a thin owner of an ``hmn_ctx*``)."""

    def __init__(self, cfg: dict, grid, precision: int = 0, ghost: int = 0):
        """ghost = 2 makes every host array carry HORMONE's two ghost layers
        per side (the Fortran module arrays' layout); 0 is packed."""
        L = lib()
        self.cfg = cfg
        n = cfg["n"]
        self.ghost = ghost
        self.shape = (n[2] + 2 * ghost, n[1] + 2 * ghost, n[0] + 2 * ghost)
        self.nvar = cfg["nvar"]
        self.nspc = int(cfg.get("nspc", 0))
        self._grid_arrays = []
        g = HmnGrid()
        for a in range(3):
            g.n[a] = n[a]
        g.ghost = ghost
        bc = np.asarray(cfg["bc"], dtype=np.int32).reshape(-1)
        for q in range(12):
            g.bc[q] = int(bc[q])
        for key in ("x", "xi", "dx", "dxi", "idx", "idxi"):
            arr = getattr(g, key)
            for a in range(3):
                v = np.ascontiguousarray(grid[a][key], dtype=np.float64)
                self._grid_arrays.append(v)
                arr[a] = _dp(v)
        p = params_struct(cfg, precision)
        h = _P()
        rc = L.hmn_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h))
        if rc != 0:
            raise HmnError(rc, "hmn_create")
        self.h = h
        if int(cfg.get("crdnt", 0)) in (1, 2):
            self.set_metric(grid, int(cfg["crdnt"]))

    def set_metric(self, grid, crdnt: int = 2):
        """Curvilinear metric factors (metric.f90:53-151) from the grid's
        ``detg``/``idetg``/``sx`` (r) and, spherical, ``sini``/``cosi``/
        ``scot``/``sinc``/``sisin`` (theta)."""
        m = HmnMetric()
        self._metric_arrays = []
        for field, a, k in (("detg1", 0, "detg"), ("idetg1", 0, "idetg"), ("sx1", 0, "sx"), ("sini", 1, "sini"),
                            ("cosi", 1, "cosi"), ("scot", 1, "scot"), ("sinc", 1, "sinc"), ("sisin", 1, "sisin")):
            if k not in grid[a]:  # the theta factors of a cylindrical grid
                continue
            v = np.ascontiguousarray(grid[a][k], dtype=np.float64)
            self._metric_arrays.append(v)
            setattr(m, field, _dp(v))
        self._check(lib().hmn_set_metric(self.h, crdnt, ctypes.byref(m)), "hmn_set_metric")

    def close(self):
        if getattr(self, "h", None):
            lib().hmn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, where):
        if rc != 0:
            cell = None
            if rc == HMN_ENEG_EINT:
                c, i, j, k, s = (ctypes.c_int() for _ in range(5))
                lib().hmn_last_error(self.h, *(ctypes.byref(x) for x in (c, i, j, k, s)))
                cell = (i.value, j.value, k.value)
            raise HmnError(rc, where, cell)

    # -- data movement -----------------------------------------------------
    def upload(self, u=None, prim=None, grvphi=None, grvpsi=None):
        keep = []

        def arr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a

        u_ = arr(u)
        pp = None
        if prim is not None:
            pp = (_DP * 9)()
            for q in range(9):
                a = arr(prim[q]) if prim[q] is not None else None
                pp[q] = _dp(a) if a is not None else _DP()
        self._check(lib().hmn_upload(self.h, _dp(u_), pp, _dp(arr(grvphi)), _dp(arr(grvpsi))), "hmn_upload")

    def download(self, prims=True, u=True, gravity=False) -> Dict[str, np.ndarray]:
        out: Dict[str, np.ndarray] = {}
        # ghosted layouts: the ghost layers are never written, leave them NaN
        new = (lambda shape: np.full(shape, np.nan)) if self.ghost else np.empty
        U = new((self.nvar,) + self.shape) if u else None
        pp = None
        if prims:
            P = new((9,) + self.shape)
            pp = (_DP * 9)()
            for q in range(9):
                pp[q] = _dp(P[q])
        gphi = new(self.shape) if gravity else None
        gpsi = new(self.shape) if gravity else None
        self._check(lib().hmn_download(self.h, _dp(U), pp, _dp(gphi), _dp(gpsi)), "hmn_download")
        if u:
            out["u"] = U
        if prims:
            for q, k in enumerate(("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")):
                out[k] = P[q]
        if gravity:
            out["grvphi"], out["grvpsi"] = gphi, gpsi
        return out

    def checkpoint_begin(self, u=True, gravity=False) -> Dict[str, np.ndarray]:
        """Start an asynchronous snapshot of the current state; the returned
        arrays are filled by checkpoint_wait (keep them alive until then)."""
        out: Dict[str, np.ndarray] = {}
        if u:
            out["u"] = np.empty((self.nvar,) + self.shape)
        P = np.empty((9,) + self.shape)
        pp = (_DP * 9)()
        for q, k in enumerate(("d", "v1", "v2", "v3", "e", "b1", "b2", "b3", "phi")):
            out[k] = P[q]
            pp[q] = _dp(P[q])
        if gravity:
            out["grvphi"], out["grvpsi"] = np.empty(self.shape), np.empty(self.shape)
        spc = np.empty(self.shape + (self.nspc,)) if self.nspc else None
        self._ck = (out, spc)
        self._check(lib().hmn_checkpoint_begin(self.h, _dp(out.get("u")), pp, _dp(out.get("grvphi")),
                                               _dp(out.get("grvpsi")), _dp(spc)), "hmn_checkpoint_begin")
        return out

    def checkpoint_wait(self) -> Dict[str, np.ndarray]:
        self._check(lib().hmn_checkpoint_wait(self.h), "hmn_checkpoint_wait")
        (out, spc), self._ck = getattr(self, "_ck", (None, None)), None
        if out is not None and spc is not None:
            out["spc"] = np.ascontiguousarray(np.moveaxis(spc, -1, 0))
        return out

    def set_flux_boundary(self, flux):
        """Boundary code 10 at the inner x3 face: its flux, 9 conserved slots
        then the scalars (fluxboundary.f90:42-87)."""
        a = np.ascontiguousarray(flux, dtype=np.float64)
        self._flux_boundary = a
        self._check(lib().hmn_set_flux_boundary(self.h, 2, 0, _dp(a)), "hmn_set_flux_boundary")

    def set_dirichlet(self, axis: int, side: int, vals: np.ndarray):
        """Ghost values of a code-9 face: (8 + nspc, 2, n_slow, n_fast) for the
        planes d, p, v1, v2, v3, b1, b2, b3, scalars."""
        a = np.ascontiguousarray(vals, dtype=np.float64)
        self._keep_dir = getattr(self, "_keep_dir", {})
        self._keep_dir[(axis, side)] = a
        self._check(lib().hmn_set_dirichlet(self.h, int(axis), int(side), _dp(a)), "hmn_set_dirichlet")

    def upload_scalars(self, spc: np.ndarray):
        """spc: (nspc, nz, ny, nx) mass fractions."""
        a = np.ascontiguousarray(np.moveaxis(np.asarray(spc, dtype=np.float64), 0, -1))
        self._check(lib().hmn_upload_scalars(self.h, _dp(a)), "hmn_upload_scalars")

    def download_scalars(self) -> np.ndarray:
        a = np.empty(self.shape + (self.nspc,))
        self._check(lib().hmn_download_scalars(self.h, _dp(a)), "hmn_download_scalars")
        return np.ascontiguousarray(np.moveaxis(a, -1, 0))

    def gravity_clock(self):
        g, c = _D(), _D()
        self._check(lib().hmn_gravity_clock(self.h, ctypes.byref(g), ctypes.byref(c)), "hmn_gravity_clock")
        return g.value, c.value

    def pressure(self) -> np.ndarray:
        p = np.empty(self.shape)
        self._check(lib().hmn_download_pressure(self.h, _dp(p)), "hmn_download_pressure")
        return p

    # -- the step loop entry points -------------------------------------------
    def timestep(self, time, t_out, t_end):
        dt, ch = _D(), _D()
        self._check(lib().hmn_timestep(self.h, float(time), float(t_out), float(t_end), ctypes.byref(dt),
                                       ctypes.byref(ch)), "hmn_timestep")
        return dt.value, ch.value

    def gravity_step(self, time, dt, tn):
        self._check(lib().hmn_gravity_step(self.h, float(time), float(dt), int(tn)), "hmn_gravity_step")

    def set_gravity_clock(self, grvtime, cgrav_old):
        self._check(lib().hmn_set_gravity_clock(self.h, float(grvtime), float(cgrav_old)), "hmn_set_gravity_clock")

    def hydro_step(self):
        self._check(lib().hmn_hydro_step(self.h), "hmn_hydro_step")

    def phidamp(self):
        self._check(lib().hmn_phidamp(self.h), "hmn_phidamp")

    def run(self, time, t_end, max_steps):
        t = _D(time)
        steps = _I(0)
        self._check(lib().hmn_run(self.h, ctypes.byref(t), float(t_end), int(max_steps), ctypes.byref(steps)),
                    "hmn_run")
        return t.value, steps.value

    def sync(self):
        self._check(lib().hmn_sync(self.h), "hmn_sync")

    EVO = ("Mtot", "Etot", "Eitot", "Ektot", "Egtot", "Mbound", "Ebound", "Jbound", "Ebtot", "Jtot")

    def evo(self) -> Dict[str, float]:
        """hmn_evo: the ten totals of evo_output (output.f90:147-275), by name."""
        out = (_D * 10)()
        self._check(lib().hmn_evo(self.h, out), "hmn_evo")
        return dict(zip(self.EVO, list(out)))

    def launches(self) -> int:
        return int(lib().hmn_launch_count(self.h))

    def stream_ptr(self) -> int:
        return int(lib().hmn_stream(self.h) or 0)


# ---------------------------------------------------------------------------
# slab decomposition along z (hmn_set_slab and friends)

def _bind_slab(L):
    if getattr(L, "_hmn_slab_bound", False):
        return L
    L.hmn_slab_halo_bytes.argtypes = [_P]
    L.hmn_slab_halo_bytes.restype = ctypes.c_size_t
    L.hmn_set_slab.argtypes = [_P, _P, _P, _P, _P, _I, _I]
    L.hmn_set_slab_push.argtypes = [_P, _P * 2, _P * 2, _P * 2, _P * 2, _I, _I]
    L.hmn_set_slab_push.restype = _I
    L.hmn_pack_halos.argtypes = [_P]
    L.hmn_hydro_stage.argtypes = [_P, _I]
    L.hmn_cfl_local.argtypes = [_P, _D, _D, _D]
    L.hmn_cfl_partials.argtypes = [_P, ctypes.POINTER(_P), ctypes.POINTER(_P)]
    L.hmn_cfl_finalize.argtypes = [_P, _DP, _DP]
    L.hmn_slab_gravity_halo_bytes.argtypes = [_P]
    L.hmn_slab_gravity_halo_bytes.restype = ctypes.c_size_t
    L.hmn_set_slab_gravity.argtypes = [_P, _P, _P, _P, _P]
    L.hmn_pack_gravity_halos.argtypes = [_P]
    L.hmn_gravity_unit.argtypes = [_P, _DP]
    L.hmn_set_gravity_unit.argtypes = [_P, _D]
    L.hmn_gravity_begin.argtypes = [_P, _D, _D, _I, ctypes.POINTER(_I)]
    L.hmn_gravity_substage.argtypes = [_P]
    for n in ("hmn_set_slab", "hmn_pack_halos", "hmn_hydro_stage", "hmn_cfl_local", "hmn_cfl_partials",
              "hmn_cfl_finalize", "hmn_set_slab_gravity", "hmn_pack_gravity_halos", "hmn_gravity_unit",
              "hmn_set_gravity_unit", "hmn_gravity_begin", "hmn_gravity_substage"):
        getattr(L, n).restype = _I
    L._hmn_slab_bound = True
    return L


class SlabContext(Context):
    """A Context for one slab of a z-decomposed grid."""

    def halo_bytes(self) -> int:
        return int(_bind_slab(lib()).hmn_slab_halo_bytes(self.h))

    def set_slab(self, send_lo, send_hi, recv_lo, recv_hi, wrap_lo=False, wrap_hi=False):
        """Device addresses (ints, 0 for a physical face) of the halo buffers;
        wrap_* mark the grid's periodic z boundary."""
        L = _bind_slab(lib())
        self._check(L.hmn_set_slab(self.h, send_lo or None, send_hi or None, recv_lo or None, recv_hi or None,
                                   int(bool(wrap_lo)), int(bool(wrap_hi))), "hmn_set_slab")

    def set_slab_push(self, recv_lo, recv_hi, push_lo, push_hi, wrap_lo=False, wrap_hi=False):
        """The push exchange: pairs (parity 0, 1) of device addresses (0 on
        a physical face) of this slab's halo buffers and of the neighbours'
        buffers its stages store into."""
        L = _bind_slab(lib())
        arr = lambda pair: (_P * 2)(*[v or None for v in pair])  # noqa: E731
        self._check(L.hmn_set_slab_push(self.h, arr(recv_lo), arr(recv_hi), arr(push_lo), arr(push_hi),
                                        int(bool(wrap_lo)), int(bool(wrap_hi))), "hmn_set_slab_push")

    def pack_halos(self):
        self._check(_bind_slab(lib()).hmn_pack_halos(self.h), "hmn_pack_halos")

    # the potential's halos and the gravity sub-stages of a slab with gravity
    def gravity_halo_bytes(self) -> int:
        return int(_bind_slab(lib()).hmn_slab_gravity_halo_bytes(self.h))

    def set_slab_gravity(self, send_lo, send_hi, recv_lo, recv_hi):
        L = _bind_slab(lib())
        self._check(L.hmn_set_slab_gravity(self.h, send_lo or None, send_hi or None, recv_lo or None,
                                           recv_hi or None), "hmn_set_slab_gravity")

    def pack_gravity_halos(self):
        self._check(_bind_slab(lib()).hmn_pack_gravity_halos(self.h), "hmn_pack_gravity_halos")

    def gravity_unit(self) -> float:
        v = _D()
        self._check(_bind_slab(lib()).hmn_gravity_unit(self.h, ctypes.byref(v)), "hmn_gravity_unit")
        return v.value

    def set_gravity_unit(self, dtg_unit: float):
        self._check(_bind_slab(lib()).hmn_set_gravity_unit(self.h, float(dtg_unit)), "hmn_set_gravity_unit")

    def gravity_begin(self, time, dt, tn) -> int:
        n = _I()
        self._check(_bind_slab(lib()).hmn_gravity_begin(self.h, float(time), float(dt), int(tn), ctypes.byref(n)),
                    "hmn_gravity_begin")
        return n.value

    def gravity_substage(self):
        self._check(_bind_slab(lib()).hmn_gravity_substage(self.h), "hmn_gravity_substage")

    def hydro_stage(self, stage: int):
        self._check(_bind_slab(lib()).hmn_hydro_stage(self.h, int(stage)), "hmn_hydro_stage")

    def cfl_local(self, time, t_out, t_end):
        self._check(_bind_slab(lib()).hmn_cfl_local(self.h, float(time), float(t_out), float(t_end)), "hmn_cfl_local")

    def cfl_partials(self):
        a, b = _P(), _P()
        self._check(_bind_slab(lib()).hmn_cfl_partials(self.h, ctypes.byref(a), ctypes.byref(b)), "hmn_cfl_partials")
        return int(a.value), int(b.value)

    def cfl_finalize(self):
        dt, ch = _D(), _D()
        self._check(_bind_slab(lib()).hmn_cfl_finalize(self.h, ctypes.byref(dt), ctypes.byref(ch)), "hmn_cfl_finalize")
        return dt.value, ch.value
