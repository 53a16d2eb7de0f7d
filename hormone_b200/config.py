"""Parameter-file driven set-up (the drop-in for HORMONE's namelist layer).

HORMONE resolves its settings in three layers (src/main/setup.f90:69-169):
``para/parameters_base`` -> ``para/parameters_<simtype>`` -> the user's
``parafile``, then derives flags in ``checksetup`` (src/main/checksetup.f90:
11-175).  This module reads the same Fortran namelist files with a small
parser and applies the same derivations, restricted to the settings the
explicit hydro/MHD/hyperbolic-gravity step uses.

The built-in defaults below restate the values of ``para/parameters_base``
and of the per-simtype files that have golden test data, so that a run needs
no copy of the reference's ``para/`` directory; a directory holding
HORMONE-format parameter files can be given instead and then takes over.
"""
from __future__ import annotations

import math
import os
import re
from typing import Any, Dict, Optional

import numpy as np

# ---------------------------------------------------------------------------
# Fortran namelist reader

_TOKEN = re.compile(r"""\s*(?:(?P<str>'[^']*'|"[^"]*")|(?P<word>[^\s,=/]+(?:\([^)]*\))?)|(?P<eq>=)|(?P<sep>,)|(?P<end>/))""")


def _convert(tok: str) -> Any:
    t = tok.strip()
    if t.startswith(("'", '"')):
        return t[1:-1]
    low = t.lower()
    if low in (".true.", ".t.", "t", "true"):
        return True
    if low in (".false.", ".f.", "f", "false"):
        return False
    if re.fullmatch(r"[+-]?\d+", t):
        return int(t)
    f = re.fullmatch(r"([+-]?(?:\d+\.?\d*|\.\d+))(?:[dDeE]([+-]?\d+))?", t)
    if f:
        mant, ex = f.group(1), f.group(2)
        return float(mant + ("e" + ex if ex else ""))
    raise ValueError(f"cannot parse namelist value {tok!r}")


def parse_namelists(text: str) -> Dict[str, Dict[str, Any]]:
    """Return {group: {key: value}} for every ``&group ... /`` block in text.

    Comments start with ``!``; keys are lower-cased (Fortran is
    case-insensitive).  Array-element keys such as ``fmr_lvl(1:20)`` are kept
    verbatim.
    """
    out: Dict[str, Dict[str, Any]] = {}
    lines = []
    for ln in text.splitlines():
        # strip comments that are not inside a string
        res, q = [], None
        for ch in ln:
            if q:
                res.append(ch)
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                res.append(ch)
            elif ch == "!":
                break
            else:
                res.append(ch)
        lines.append("".join(res))
    body = "\n".join(lines)
    for m in re.finditer(r"&(\w+)(.*?)(?:/|(?=&)|\Z)", body, flags=re.S):
        group = m.group(1).lower()
        content = m.group(2)
        vals: Dict[str, Any] = {}
        toks = [mm for mm in _TOKEN.finditer(content) if mm.group(0).strip()]
        i = 0
        while i < len(toks):
            t = toks[i]
            if t.group("word") and i + 1 < len(toks) and toks[i + 1].group("eq"):
                key = t.group("word").lower()
                j = i + 2
                items = []
                while j < len(toks) and not (toks[j].group("word") and j + 1 < len(toks) and toks[j + 1].group("eq")):
                    if toks[j].group("str") or toks[j].group("word"):
                        items.append(_convert(toks[j].group(0)))
                    j += 1
                vals[key] = items[0] if len(items) == 1 else items
                i = j
            else:
                i += 1
        out.setdefault(group, {}).update(vals)
    return out


# ---------------------------------------------------------------------------
# built-in defaults (para/parameters_base and the golden-test simtypes)

BASE: Dict[str, Any] = dict(
    xi1s=0.0, xi1e=1.0, xi2s=0.0, xi2e=1.0, xi3s=0.0, xi3e=1.0,
    is_=1, ie=10, js=1, je=1, ks=1, ke=1, imesh=0, jmesh=0, kmesh=0, x1min=0.0, x2min=0.0, x3min=0.0,
    outstyle=1, endstyle=1, tnlim=0, t_end=0.0, dt_out=1.0, tn_out=1, dt_unit="s",
    eostype=0, compswitch=0, muconst=0.62, spn=0, gamma=1.6666666666666667,
    crdnt=0, courant=0.9, rktype=3, mag_on=False, flux_limiter="modified_mc", alpha9wave=0.1,
    bc1is=0, bc1os=0, bc2is=0, bc2os=0, bc3is=0, bc3os=0,
    bc1iv=0, bc1ov=0, bc2iv=0, bc2ov=0, bc3iv=0, bc3ov=0,
    gravswitch=0, HGfac=5.0, hgcfl=0.9, maxtngrv=-1, gbtype=0, grktype=2, alphagrv=0.1,
    G=6.67430e-8, fixed_dt=-1.0, eq_sym=False,
    test_tol=1e-15, Mach_tol=1e-5,
)

_TUBE_TIMES = dict(outstyle=1, endstyle=1, tnlim=100000, t_end=200.0, dt_out=200.0, tn_out=1, dt_unit="ms")

SIMTYPES: Dict[str, Dict[str, Any]] = {
    # para/parameters_sodshock_{x,y,z}
    "sodshock_x": dict(ie=500, gamma=1.4, bc1is=3, bc1os=3, bc1iv=3, bc1ov=3, **_TUBE_TIMES),
    "sodshock_y": dict(ie=1, je=500, gamma=1.4, bc2is=3, bc2os=3, bc2iv=3, bc2ov=3, **_TUBE_TIMES),
    "sodshock_z": dict(ie=1, ke=500, gamma=1.4, bc3is=3, bc3os=3, bc3iv=3, bc3ov=3, **_TUBE_TIMES),
    # para/parameters_briowushock_{x,y,z}
    "briowushock_x": dict(ie=500, gamma=2.0, mag_on=True, bc1is=3, bc1os=3, bc1iv=3, bc1ov=3, **_TUBE_TIMES),
    "briowushock_y": dict(ie=1, je=500, gamma=2.0, mag_on=True, bc2is=3, bc2os=3, bc2iv=3, bc2ov=3, **_TUBE_TIMES),
    "briowushock_z": dict(ie=1, ke=500, gamma=2.0, mag_on=True, bc3is=3, bc3os=3, bc3iv=3, bc3ov=3, **_TUBE_TIMES),
    # para/parameters_orszagtang_{xy,yz,xz}
    "orszagtang_xy": dict(ie=128, je=128, mag_on=True, outstyle=1, endstyle=1, tnlim=100000, t_end=500.0,
                          dt_out=500.0, tn_out=1, dt_unit="ms", test_tol=7e-15),
    "orszagtang_yz": dict(ie=1, je=128, ke=128, mag_on=True, outstyle=1, endstyle=1, tnlim=100000, t_end=500.0,
                          dt_out=500.0, tn_out=1, dt_unit="ms", test_tol=7e-15),
    "orszagtang_xz": dict(ie=128, ke=128, mag_on=True, outstyle=1, endstyle=1, tnlim=100000, t_end=500.0,
                          dt_out=500.0, tn_out=1, dt_unit="ms", test_tol=7e-15),
    # para/parameters_sedov_default (spherical, 1-D radial) with
    # para/extras_sedov (gamma=1.4, damb=1, Eexp=1; read by sedov.f90:30-38)
    "sedov_default": dict(xi1s=0.0, xi1e=1.0, ie=500, outstyle=1, endstyle=1, tnlim=100000, t_end=300.0,
                          dt_out=300.0, tn_out=1, dt_unit="ms", eostype=0, crdnt=2, flux_limiter="modified_mc",
                          bc1is=1, bc1os=2, bc1iv=1, bc1ov=2, test_tol=2e-14, gamma=1.4, damb=1.0, Eexp=1.0),
    # para/parameters_KHinstability (two passive scalars)
    "KHinstability": dict(xi1s=-0.5, xi1e=0.5, xi2s=-0.5, xi2e=0.5, ie=128, je=128, outstyle=1, endstyle=1,
                          tnlim=100000, t_end=1000.0, dt_out=100.0, tn_out=1, dt_unit="ms", compswitch=2, spn=2),
}

_UNITS = {"yr": 3600.0 * 24.0 * 365.25, "d": 3600 * 24.0, "hr": 3600.0, "ks": 1000.0, "min": 60.0, "s": 1.0,
          "ms": 1e-3, "ns": 1e-9}

_LIMITERS = {"flat": 0, "minmod": 1, "modified_mc": 2}


def _flatten(groups: Dict[str, Dict[str, Any]]) -> Dict[str, Any]:
    flat: Dict[str, Any] = {}
    for g in groups.values():
        for k, v in g.items():
            key = "is_" if k == "is" else k
            # keep the case of the names that the defaults use
            for dk in BASE:
                if dk.lower() == key:
                    key = dk
                    break
            flat[key] = v
    return flat


def read_parameter_file(path: str) -> Dict[str, Any]:
    with open(path) as fh:
        return _flatten(parse_namelists(fh.read()))


def resolve(simtype: str, parafile: Optional[str] = None, para_dir: Optional[str] = None,
            overrides: Optional[Dict[str, Any]] = None, is_test: bool = False) -> Dict[str, Any]:
    """Resolve the settings of a run and apply checksetup's derivations.

    ``simtype`` may end in `` test`` (setup.f90:44-56), which sets
    ``is_test`` and ignores ``parafile``.
    """
    st = simtype.strip()
    if st.endswith(" test"):
        st, is_test = st[:-5].strip(), True
    raw: Dict[str, Any] = dict(BASE)
    base_file = os.path.join(para_dir, "parameters_base") if para_dir else None
    if base_file and os.path.exists(base_file):
        raw.update(read_parameter_file(base_file))
    sim_file = os.path.join(para_dir, f"parameters_{st}") if para_dir else None
    if sim_file and os.path.exists(sim_file):
        raw.update(read_parameter_file(sim_file))
    elif st in SIMTYPES:
        raw.update(SIMTYPES[st])
    if parafile and not is_test:
        raw.update(read_parameter_file(parafile))
    if overrides:
        raw.update(overrides)
    raw["simtype"] = st
    raw["is_test"] = is_test
    return checksetup(raw)


def checksetup(raw: Dict[str, Any]) -> Dict[str, Any]:
    """Derived settings of src/main/checksetup.f90:24-209 for this path."""
    cfg = dict(raw)
    is_, ie, js, je, ks, ke = (int(cfg[k]) for k in ("is_", "ie", "js", "je", "ks", "ke"))
    if ie < is_ or je < js or ke < ks:
        raise ValueError("grid indices must satisfy ie>=is, je>=js, ke>=ks")
    n = [ie - is_ + 1, je - js + 1, ke - ks + 1]
    solve = [ie > is_, je > js, ke > ks]
    dim = sum(solve)
    if dim == 0:
        raise ValueError("Error from gridset: no direction to solve")
    crdnt = int(cfg.get("crdnt", 0))
    if crdnt not in (0, 1, 2):
        raise ValueError("Cartesian (0), cylindrical (1) and spherical (2) coordinates are on this path")
    if crdnt == 1 and n[1] != 1:
        raise ValueError("cylindrical grids with a solved phi axis are not on this path (gridset reads an unset "
                         "width for their phi ghosts); use one phi cell (axisymmetric R-z)")
    if int(cfg.get("eostype", 0)) != 0:
        raise ValueError("only the ideal-gas EOS (eostype=0) is on this path")
    mag_on = bool(cfg["mag_on"])
    glm = mag_on and dim > 1
    nvar = 5 + (3 if mag_on else 0) + (1 if glm else 0)
    bc = np.zeros((3, 2, 2), dtype=np.int32)
    for a in range(3):
        for io, tag in enumerate(("i", "o")):
            for sv, kind in enumerate(("s", "v")):
                bc[a, io, sv] = int(cfg[f"bc{a + 1}{tag}{kind}"])
    for a in range(3):
        for sv in range(2):
            x, y = bc[a, 0, sv], bc[a, 1, sv]
            if x * y == 0 and x + y != 0:
                raise ValueError(f"boundary condition axis {a + 1}: both sides must be periodic")
    if crdnt == 1:  # periodic phi (checksetup.f90:110-111)
        bc[1] = 0
    if crdnt == 2:  # polar boundaries (checksetup.f90:112-115, :134-137)
        bc[1] = 1
        bc[2] = 0
    if not solve[0]:
        bc[0] = 2
    if not solve[1]:
        bc[1] = 3
    if not solve[2]:
        bc[2] = 3
    for a in range(3):
        if solve[a]:
            for io in range(2):
                for code in bc[a, io]:
                    if code == 10 and a == 2 and io == 0 and bc[2, 0, 0] == bc[2, 0, 1] == 10:
                        continue  # the flux boundary exists at the inner x3 face only (fluxboundary.f90:22-28)
                    if code not in (0, 1, 2, 3, 4, 5, 9):
                        raise ValueError(f"boundary code {code} on axis {a + 1} is not supported on this path")
    if float(cfg["courant"]) > 1.0:
        raise ValueError("courant number should be <= 1.0")
    unit = _UNITS[str(cfg["dt_unit"])]
    dt_out = float(cfg["dt_out"]) * unit
    t_end = float(cfg["t_end"]) * unit
    t_out = min(dt_out, t_end)
    tn_out = int(cfg["tn_out"])
    if cfg.get("is_test"):
        t_out = t_end
        tn_out = int(cfg["tnlim"])
    lim = str(cfg["flux_limiter"])
    if lim not in _LIMITERS:
        raise ValueError(f"Error in flux_limiter {lim}")
    comp = int(cfg.get("compswitch", 0))
    if comp not in (0, 1, 2):
        raise ValueError(f"Error in compswitch {comp}")
    # passive scalars are carried with compswitch 2 (compswitch 1 only changes
    # the mean molecular weight, which the ideal-gas step does not use)
    nspc = int(cfg.get("spn", 0)) if comp == 2 else 0
    if nspc < 0 or nspc > 8:
        raise ValueError("at most 8 passive scalars are on this path")
    if crdnt and nspc:
        raise ValueError("passive scalars on curvilinear grids are not on this path")
    grav = int(cfg.get("gravswitch", 0))
    if crdnt == 1 and grav:
        raise ValueError("self-gravity on cylindrical grids is not on this path")
    if crdnt == 2 and grav:
        # setup_grv_hyperbolic (gravity_hyperbolic.f90:336-405) has spherical
        # coefficients for (r, theta) with one phi cell and for 3-D grids; the
        # outer radius takes the Robin condition (gbtype 1) here
        if grav != 3 or not (solve[0] and solve[1]):
            raise ValueError("spherical self-gravity needs gravswitch 3 on an (r, theta) or 3-D grid")
        if int(cfg.get("gbtype", 0)) != 1:
            raise ValueError("spherical self-gravity takes the Robin outer boundary (gbtype=1) on this path")
    if grav not in (0, 3):
        raise ValueError("only gravswitch 0 (off) or 3 (hyperbolic) is on this path")
    if grav == 3 and dim != 3 and crdnt == 0:
        raise ValueError("the Cartesian hyperbolic gravity solver needs a 3-D grid")
    extent = [(float(cfg["xi1s"]), float(cfg["xi1e"])), (float(cfg["xi2s"]), float(cfg["xi2e"])),
              (float(cfg["xi3s"]), float(cfg["xi3e"]))]
    if crdnt == 2:  # gridset.f90:295-296
        half = n[1] == 1 or bool(cfg.get("eq_sym", False))
        extent[1] = (0.0, math.pi * 0.5 if half else math.pi)
        extent[2] = (-math.pi, math.pi)
    if crdnt == 1:  # a quarter turn of phi for one phi cell (gridset.f90:209-231)
        extent[1] = (extent[1][0], extent[1][0] + 2.0 * math.pi / 4.0)
    cfg.update(
        n=n, solve=solve, dim=dim, mag_on=mag_on, glm=glm, nvar=nvar, bc=bc, crdnt=crdnt,
        extent=extent,
        t_end=t_end, dt_out=dt_out, t_out=t_out, tn_out=tn_out, limiter_code=_LIMITERS[lim],
        rktype=int(cfg["rktype"]), gamma=float(cfg["gamma"]), courant=float(cfg["courant"]),
        alpha9wave=float(cfg["alpha9wave"]), outstyle=int(cfg["outstyle"]), endstyle=int(cfg["endstyle"]),
        tnlim=int(cfg["tnlim"]), gravswitch=grav, HGfac=float(cfg["HGfac"]), hgcfl=float(cfg["hgcfl"]),
        alphagrv=float(cfg["alphagrv"]), G=float(cfg["G"]), grktype=int(cfg["grktype"]),
        maxtngrv=int(cfg["maxtngrv"]), compswitch=comp, nspc=nspc,
    )
    return cfg
