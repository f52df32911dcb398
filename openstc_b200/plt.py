"""Reader and writer of the binary Tecplot V112 flow-field file in the layout
the reference writes (src/MPIIO.hpp:59-546): ordered zones, FP64 data,
interior points only."""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np


def _str(s: str) -> bytes:
    return b"".join(struct.pack("<i", ord(c)) for c in s) + struct.pack("<i", 0)


def write_plt(path: str | Path, names: list[str], zones: list[dict[str, np.ndarray]]) -> None:
    """zones: one dict per block mapping variable name -> array (nz, ny, nx)."""
    out = bytearray()
    out += b"#!TDV112" + struct.pack("<ii", 1, 0) + _str("Solution file") + struct.pack("<i", len(names))
    for n in names:
        out += _str(n)
    for z, zone in enumerate(zones):
        nz, ny, nx = zone[names[0]].shape
        out += struct.pack("<f", 299.0) + _str(f"zone {z}")
        out += struct.pack("<iidiiiiiiiii", -1, -2, 0.0, -1, 0, 0, 0, 0, nx, ny, nz, 0)
    out += struct.pack("<f", 357.0)
    for zone in zones:
        out += struct.pack("<f", 299.0) + struct.pack(f"<{len(names)}i", *([2] * len(names)))
        out += struct.pack("<iii", 0, 0, -1)
        for n in names:
            a = zone[n]
            out += struct.pack("<dd", float(a.min()), float(a.max()))
        for n in names:
            out += np.ascontiguousarray(zone[n], dtype="<f8").tobytes()
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    Path(path).write_bytes(bytes(out))


def read_plt(path: str | Path) -> tuple[list[str], list[dict[str, np.ndarray]]]:
    buf = Path(path).read_bytes()
    pos = 16

    def i32():
        nonlocal pos
        v = struct.unpack_from("<i", buf, pos)[0]
        pos += 4
        return v

    def sstr():
        chars = []
        while True:
            c = i32()
            if c == 0:
                return "".join(chars)
            chars.append(chr(c))

    if buf[:8] != b"#!TDV112":
        raise ValueError(f"{path} is not a Tecplot V112 file")
    sstr()
    nvar = i32()
    names = [sstr() for _ in range(nvar)]
    dims = []
    while True:
        marker = struct.unpack_from("<f", buf, pos)[0]
        pos += 4
        if marker == 357.0:
            break
        sstr()
        pos += 36
        nx, ny, nz = i32(), i32(), i32()
        pos += 4
        dims.append((nz, ny, nx))
    zones = []
    for nz, ny, nx in dims:
        pos += 4 + 4 * nvar + 12 + 16 * nvar
        npt = nx * ny * nz
        zone = {}
        for n in names:
            zone[n] = np.frombuffer(buf, dtype="<f8", count=npt, offset=pos).reshape(nz, ny, nx).copy()
            pos += 8 * npt
        zones.append(zone)
    return names, zones
