"""ORACLE (test infrastructure only): numpy restatement of the reference's
restart file layout (read_write.f90:16-40 write_params / sav_field /
read_field, opened as Fortran unformatted sequential files in
les.F90:69-82 and 331-351): each record framed by its byte length as a
4-byte integer; reals of real_bytes (4 shipped, 8 with -fdefault-real-8),
integers of 4 bytes.

  record 1: time, nnx, nny, nnz, xl, yl, zl
  record 2: dt, z0, utau
  record 3: divgls, fcor, ugtop, ugbot, vgtop, vgbot
  record 3+iz: u, v, w, e, p(1:nnx,1:nny) of level iz, iz = 1..nnz
Fields are (nnz, nny, nnx) arrays (x fastest).
"""
import struct

import numpy as np


def _rec(fh, payload):
    fh.write(struct.pack("<i", len(payload)))
    fh.write(payload)
    fh.write(struct.pack("<i", len(payload)))


def write_field(path, fields, header, real_bytes=8):
    """fields: dict u, v, w, e, p; header: dict time, xl, yl, zl, dt, z0,
    utau (divgls .. vgbot default 0)."""
    rt = "<d" if real_bytes == 8 else "<f"
    dt = np.float64 if real_bytes == 8 else np.float32
    nz, ny, nx = fields["u"].shape
    with open(path, "wb") as fh:
        _rec(fh, struct.pack(rt, header["time"]) + struct.pack("<3i", nx, ny, nz) +
             b"".join(struct.pack(rt, header[k]) for k in ("xl", "yl", "zl")))
        _rec(fh, b"".join(struct.pack(rt, header[k]) for k in ("dt", "z0", "utau")))
        _rec(fh, b"".join(struct.pack(rt, header.get(k, 0.0))
                          for k in ("divgls", "fcor", "ugtop", "ugbot", "vgtop", "vgbot")))
        for iz in range(nz):
            _rec(fh, b"".join(np.ascontiguousarray(fields[k][iz], dtype=dt).tobytes() for k in "uvwep"))


def read_field(path, real_bytes=8):
    """-> (header dict, fields dict)."""
    rt = "<d" if real_bytes == 8 else "<f"
    dt = np.float64 if real_bytes == 8 else np.float32
    with open(path, "rb") as fh:
        data = fh.read()
    pos = 0
    recs = []
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        recs.append(data[pos + 4:pos + 4 + n])
        (m,) = struct.unpack_from("<i", data, pos + 4 + n)
        assert m == n, "record markers differ"
        pos += 8 + n
    r1, r2, r3 = recs[:3]
    rb = real_bytes
    h = {"time": struct.unpack_from(rt, r1, 0)[0]}
    nx, ny, nz = struct.unpack_from("<3i", r1, rb)
    for i, k in enumerate(("xl", "yl", "zl")):
        h[k] = struct.unpack_from(rt, r1, rb + 12 + i * rb)[0]
    for i, k in enumerate(("dt", "z0", "utau")):
        h[k] = struct.unpack_from(rt, r2, i * rb)[0]
    for i, k in enumerate(("divgls", "fcor", "ugtop", "ugbot", "vgtop", "vgbot")):
        h[k] = struct.unpack_from(rt, r3, i * rb)[0]
    h["nnx"], h["nny"], h["nnz"] = nx, ny, nz
    assert len(recs) == 3 + nz
    f = {k: np.zeros((nz, ny, nx), dtype=dt) for k in "uvwep"}
    for iz in range(nz):
        a = np.frombuffer(recs[3 + iz], dtype=dt).reshape(5, ny, nx)
        for q, k in enumerate("uvwep"):
            f[k][iz] = a[q]
    return h, f
