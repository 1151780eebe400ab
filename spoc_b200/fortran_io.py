"""init.bin / temp.bin: the reference's Fortran sequential unformatted state files.

Layout (src/shwwnl.f:180-188 read, :309-317 and :325-333 write;
src/init.f:266-274): seven records, each framed by 4-byte little-endian record
lengths, as gfortran writes them:
    time                     (1 double)
    ((u(j,i), j=1,nm), i=1,ne)
    v, h, w, z, hb           (same, packed with stride nm, not nnmod)
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

FIELDS = ("u", "v", "h", "w", "z", "hb")


def _record(buf: bytes) -> bytes:
    n = struct.pack("<i", len(buf))
    return n + buf + n


def write_state(path: str | Path, time: float, nm: int, **fields: np.ndarray) -> None:
    """Write time and the six fields (each (ne, ld), first nm columns used)."""
    out = [_record(struct.pack("<d", float(time)))]
    for name in FIELDS:
        a = np.asarray(fields[name], dtype="<f8")[:, :nm]
        out.append(_record(np.ascontiguousarray(a).tobytes()))
    Path(path).write_bytes(b"".join(out))


def read_state(path: str | Path, nm: int) -> tuple[float, dict]:
    """Return (time, {u, v, h, w, z, hb}) with arrays of shape (ne, nm)."""
    data = Path(path).read_bytes()
    pos, recs = 0, []
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        body = data[pos + 4: pos + 4 + n]
        (m,) = struct.unpack_from("<i", data, pos + 4 + n)
        if m != n or len(body) != n:
            raise ValueError(f"{path}: corrupt record at byte {pos}")
        recs.append(body)
        pos += 8 + n
    if len(recs) != 1 + len(FIELDS):
        raise ValueError(f"{path}: expected 7 records, found {len(recs)}")
    (time,) = struct.unpack("<d", recs[0])
    out = {}
    for name, body in zip(FIELDS, recs[1:]):
        a = np.frombuffer(body, dtype="<f8")
        if a.size % nm:
            raise ValueError(f"{path}: record {name} is not a multiple of nm={nm}")
        out[name] = a.reshape(-1, nm).astype(np.float64)
    return time, out


def fortran_e(v: float, w: int = 10, d: int = 3) -> str:
    """Fortran Ew.d edit descriptor as gfortran writes it: 0.ddd mantissa,
    E+ee exponent (three-digit exponents drop the E), right-justified."""
    import math
    if math.isnan(v):
        return "NaN".rjust(w)
    if math.isinf(v):
        return ("-Infinity" if v < 0 else "Infinity").rjust(w)
    neg = math.copysign(1.0, v) < 0
    if v == 0.0:
        digits, exp = "0" * d, 0
    else:
        s = f"{abs(v):.{d - 1}e}"
        mant, e = s.split("e")
        digits = mant.replace(".", "")
        exp = int(e) + 1
    body = f"0.{digits}E{exp:+03d}" if abs(exp) <= 99 else f"0.{digits}{exp:+04d}"
    return (("-" if neg else "") + body).rjust(w)


def gra_name(name: str, nper: int) -> str:
    """write_gra's file name (src/visu2.f:102-110): field letter, output number, '.gra'."""
    return f"{name}{nper:d}.gra"


def write_gra(path: str | Path, lattice: np.ndarray, field: int) -> None:
    """write_gra (src/visu2.f:86-149): one line 'x y value' per lattice point
    of every element in format 3(e10.3,1x).  lattice is (ne, np, 5) from
    Solver.lattice (x, y, u, v, h); field 0, 1, 2 selects u, v, h."""
    lines = []
    for el in lattice:
        for x, y, *vals in el:
            lines.append(f"{fortran_e(x)} {fortran_e(y)} {fortran_e(vals[field])} ")
    Path(path).write_text("\n".join(lines) + "\n")
