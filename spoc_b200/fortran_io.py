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
