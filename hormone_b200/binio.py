"""HORMONE binary dump format: reader and writer.

The layout is Fortran stream access (src/main/io.F90), written block by block
by ``write_bin`` (src/main/output.f90:697-795) and read back by ``readbin``
(src/main/readbin.f90:16-115):

    marker(int4=-1) tn(int4) time(f8) marker
    marker d v1 v2 v3 e marker                      (each n cells, i fastest)
    [marker grvphi marker]                           gravswitch>=2
    [marker grvpsi cgrav_old(f8) marker]             gravswitch==3
    [marker spn(int4) spc(spn,i,j,k) species(10-char * spn) marker]  compswitch>=2
    [marker b1 b2 b3 phi marker]                     mag_on
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

MARK = np.int32(-1)


class _Reader:
    def __init__(self, buf: bytes):
        self.b = buf
        self.o = 0

    def i4(self):
        v = int(np.frombuffer(self.b, "<i4", 1, self.o)[0])
        self.o += 4
        return v

    def f8(self):
        v = float(np.frombuffer(self.b, "<f8", 1, self.o)[0])
        self.o += 8
        return v

    def arr(self, count):
        v = np.frombuffer(self.b, "<f8", count, self.o).copy()
        self.o += 8 * count
        return v

    def marker(self):
        m = self.i4()
        if m != -1:
            raise ValueError(f"bad record marker {m} at offset {self.o - 4}")


def readbin(path_or_bytes, n, mag_on: bool, gravswitch: int = 0, compswitch: int = 0) -> Dict[str, object]:
    """Read a dump; ``n`` = (nx, ny, nz).  Arrays come back as (nz, ny, nx)."""
    buf = path_or_bytes if isinstance(path_or_bytes, (bytes, bytearray)) else open(path_or_bytes, "rb").read()
    r = _Reader(buf)
    nx, ny, nz = n
    N = nx * ny * nz
    shape = (nz, ny, nx)
    out: Dict[str, object] = {}
    r.marker(); out["tn"] = r.i4(); out["time"] = r.f8(); r.marker()
    r.marker()
    for k in ("d", "v1", "v2", "v3", "e"):
        out[k] = r.arr(N).reshape(shape)
    r.marker()
    if gravswitch >= 2:
        r.marker(); out["grvphi"] = r.arr(N).reshape(shape); r.marker()
    if gravswitch == 3:
        r.marker(); out["grvpsi"] = r.arr(N).reshape(shape); out["cgrav_old"] = r.f8(); r.marker()
    if compswitch >= 2:
        r.marker()
        spn = r.i4()
        out["spc"] = r.arr(spn * N).reshape(nz, ny, nx, spn)
        names = r.b[r.o:r.o + 10 * spn]
        r.o += 10 * spn
        out["species"] = [names[10 * s:10 * s + 10].decode("ascii", "replace").strip() for s in range(spn)]
        r.marker()
    if mag_on:
        r.marker()
        for k in ("b1", "b2", "b3", "phi"):
            out[k] = r.arr(N).reshape(shape)
        r.marker()
    if r.o != len(buf):
        raise ValueError(f"{len(buf) - r.o} trailing bytes: settings do not match the dump")
    return out


def writebin(path: Optional[str], tn: int, time: float, fields: Dict[str, np.ndarray], mag_on: bool,
             gravswitch: int = 0, cgrav_old: float = 0.0, species=None) -> bytes:
    """Write a dump in the layout above; returns the bytes (and writes them
    to ``path`` if given).  With ``fields['spc']`` ((spn, nz, ny, nx) mass
    fractions) the compswitch>=2 block is written, with ``species`` names
    (10 characters each, default scalar1, scalar2, ...)."""
    parts = []

    def mark():
        parts.append(MARK.tobytes())

    def arr(a):
        parts.append(np.ascontiguousarray(a, dtype="<f8").tobytes())

    mark(); parts.append(np.int32(tn).tobytes()); parts.append(np.float64(time).tobytes()); mark()
    mark()
    for k in ("d", "v1", "v2", "v3", "e"):
        arr(fields[k])
    mark()
    if gravswitch >= 2:
        mark(); arr(fields["grvphi"]); mark()
    if gravswitch == 3:
        mark(); arr(fields["grvpsi"]); parts.append(np.float64(cgrav_old).tobytes()); mark()
    if fields.get("spc") is not None:
        spc = np.asarray(fields["spc"], dtype="<f8")
        spn = spc.shape[0]
        names = species or [f"scalar{n + 1}" for n in range(spn)]
        mark(); parts.append(np.int32(spn).tobytes()); arr(np.moveaxis(spc, 0, -1))
        parts.append(b"".join(nm.encode("ascii")[:10].ljust(10) for nm in names)); mark()
    if mag_on:
        mark()
        for k in ("b1", "b2", "b3", "phi"):
            arr(fields[k])
        mark()
    data = b"".join(parts)
    if path:
        with open(path, "wb") as fh:
            fh.write(data)
    return data
