"""A minimal reader for the geometry files of the reference's simulations
(``simulations/input_geos/*.jld2``, written by Julia's JLD2 0.1 on Julia 1.7).

JLD2 files are HDF5 files; this reader implements the small subset of the
HDF5 format those files use (no HDF5 library is needed): a version-2
superblock, version-2 object headers ("OHDR", with "OCHK" continuation
blocks), link messages of the root group, and datasets of 64-bit IEEE floats
or 64-bit integers with compact or contiguous layout.  It returns every such
dataset of the root group by name — for the geometry files ``rvec0``, ``xc``,
``yc`` (and ``areafrac``, ``seed``), the circle packing that
ErosionPackage/src/Main.jl:37-45 loads.  Datasets of other types (the Julia
struct vectors) are skipped.
"""
from __future__ import annotations

import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"


class JLD2Error(ValueError):
    pass


def _u(b: bytes, off: int, n: int) -> int:
    return int.from_bytes(b[off:off + n], "little")


def _messages(buf: bytes, addr: int):
    """Yields (type, data) of the messages of the object header at addr,
    following continuation messages."""
    if buf[addr:addr + 4] != b"OHDR":
        raise JLD2Error(f"no object header at {addr}")
    ver, flags = buf[addr + 4], buf[addr + 5]
    if ver != 2:
        raise JLD2Error(f"object header version {ver}")
    p = addr + 6
    if flags & 0x20:
        p += 16                      # access/modification/change/birth times
    if flags & 0x10:
        p += 4                       # attribute phase change values
    size_len = 1 << (flags & 3)
    chunk = _u(buf, p, size_len)
    p += size_len
    blocks = [(p, p + chunk)]
    track_order = bool(flags & 0x04)
    while blocks:
        start, end = blocks.pop(0)
        q = start
        while q + 4 <= end - 4 + 4 and q < end:
            if end - q < 4:
                break
            mtype = buf[q]
            msize = _u(buf, q + 1, 2)
            q += 4
            if track_order:
                q += 2
            data = buf[q:q + msize]
            q += msize
            if mtype == 0x10:        # continuation: address, length of an OCHK block
                caddr, clen = _u(data, 0, 8), _u(data, 8, 8)
                if buf[caddr:caddr + 4] != b"OCHK":
                    raise JLD2Error("bad continuation block")
                blocks.append((caddr + 4, caddr + clen - 4))
            elif mtype != 0:
                yield mtype, data


def _links(buf: bytes, addr: int) -> dict:
    out = {}
    for mtype, d in _messages(buf, addr):
        if mtype != 0x06:
            continue
        flags = d[1]
        p = 2
        ltype = 0
        if flags & 0x08:
            ltype = d[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nlen_size = 1 << (flags & 3)
        nlen = _u(d, p, nlen_size)
        p += nlen_size
        name = d[p:p + nlen].decode("utf-8")
        p += nlen
        if ltype == 0:
            out[name] = _u(d, p, 8)
    return out


def _dataset(buf: bytes, addr: int):
    dims = None
    dtype = None
    raw = None
    for mtype, d in _messages(buf, addr):
        if mtype == 0x01:            # dataspace
            ver, rank, flags = d[0], d[1], d[2]
            p = 4 if ver == 2 else 8
            if ver == 2 and d[3] == 0:
                dims = ()
            dims = tuple(_u(d, p + 8 * i, 8) for i in range(rank))
        elif mtype == 0x03:          # datatype
            cls = d[0] & 0x0F
            size = _u(d, 4, 4)
            if cls == 1 and size == 8:
                dtype = np.dtype("<f8")
            elif cls == 0 and size == 8:
                signed = bool(d[1] & 0x08)
                dtype = np.dtype("<i8" if signed else "<u8")
        elif mtype == 0x08:          # data layout
            ver, lclass = d[0], d[1]
            if ver < 3:
                return None
            if lclass == 0:          # compact
                n = _u(d, 2, 2)
                raw = d[4:4 + n]
            elif lclass == 1:        # contiguous
                a, n = _u(d, 2, 8), _u(d, 10, 8)
                raw = buf[a:a + n] if a != 0xFFFFFFFFFFFFFFFF else b""
            else:
                return None
    if dtype is None or raw is None or dims is None:
        return None
    count = int(np.prod(dims)) if dims else 1
    arr = np.frombuffer(raw[:count * dtype.itemsize], dtype=dtype).copy()
    return arr if dims else arr[0]


def read(path: str) -> dict:
    """{name: numpy array or scalar} for the numeric datasets of the root group."""
    buf = open(path, "rb").read()
    base = buf.find(SIG)
    if base < 0:
        raise JLD2Error("not an HDF5/JLD2 file")
    sb = buf[base:]
    ver = sb[8]
    if ver not in (2, 3):
        raise JLD2Error(f"superblock version {ver}")
    if sb[9] != 8 or sb[10] != 8:
        raise JLD2Error("only 8-byte offsets and lengths are supported")
    # base address, extension, end of file, root object header (relative to base)
    root = _u(sb, 12 + 24, 8)
    # JLD2 writes the HDF5 part after a 512-byte text header and records that
    # offset as the base address; object and data addresses are relative to it
    view = buf[_u(sb, 12, 8):]
    out = {}
    for name, addr in _links(view, root).items():
        try:
            v = _dataset(view, addr)
        except JLD2Error:
            v = None
        if v is not None:
            out[name] = v
    return out


def circles(path: str):
    """(radii, xc, yc) of a reference geometry file (Main.jl:37-45 reads
    rvec, xc, yc the same way)."""
    d = read(path)
    r = d.get("rvec0", d.get("rvec"))
    if r is None or "xc" not in d or "yc" not in d:
        raise JLD2Error(f"{path}: no rvec0/xc/yc datasets (found {sorted(d)})")
    return np.asarray(r, float), np.asarray(d["xc"], float), np.asarray(d["yc"], float)
