"""Fortran unformatted sequential records, as the Intel and GNU Fortran runtimes lay them out.

TEST INFRASTRUCTURE ONLY: the checker of the device path's backup writer and reader
(the reference's particlesNNN.bak, main.f90:1102-1139 and restart.f90:48-149).

A record is one or more subrecords; each subrecord is a 4-byte little-endian length, the
data, and the length again.  A record longer than ``max_sub`` bytes (2^31 - 9 in the
runtimes) is split: the leading marker of every subrecord but the last is negative, the
trailing marker of every subrecord but the first is negative.
"""
from __future__ import annotations

import struct

MAX_SUB = 2147483639


def write_record(f, data: bytes, max_sub: int = MAX_SUB):
    n = len(data)
    if n == 0:
        f.write(struct.pack("<ii", 0, 0))
        return
    pos, first = 0, True
    while pos < n:
        k = min(max_sub, n - pos)
        last = pos + k == n
        f.write(struct.pack("<i", k if last else -k))
        f.write(data[pos:pos + k])
        f.write(struct.pack("<i", k if first else -k))
        pos += k
        first = False


def read_record(f) -> bytes:
    out = []
    first = True
    while True:
        h = f.read(4)
        if len(h) < 4:
            raise EOFError("no record")
        (lead,) = struct.unpack("<i", h)
        k = abs(lead)
        out.append(f.read(k))
        (tail,) = struct.unpack("<i", f.read(4))
        if abs(tail) != k or (tail < 0) == first:
            raise ValueError("bad trailing marker")
        first = False
        if lead >= 0:
            return b"".join(out)


def read_backup(path: str, ntype: int):
    """(time, gtype, Pabs_cor, np_tot[nproc][ntype], [species][...] list of (n, 6) arrays)."""
    import numpy as np
    with open(path, "rb") as f:
        time, gtype, pc = struct.unpack("<did", read_record(f))
        np_tot = np.frombuffer(read_record(f), dtype="<i4").reshape(-1, ntype)
        parts = [[] for _ in range(ntype)]
        for p in range(np_tot.shape[0]):
            for s in range(ntype):
                parts[s].append(np.frombuffer(read_record(f), dtype="<f8").reshape(-1, 6))
        rest = f.read()
    if rest:
        raise ValueError("trailing bytes")
    return time, gtype, pc, np_tot, parts


def write_backup(path: str, time: float, gtype: int, pc: float, blocks, max_sub: int = MAX_SUB):
    """blocks[iproc][ptype] = (n, 6) float64 arrays."""
    import numpy as np
    ntype = len(blocks[0])
    np_tot = np.array([[len(blocks[p][s]) for s in range(ntype)] for p in range(len(blocks))], dtype="<i4")
    with open(path, "wb") as f:
        write_record(f, struct.pack("<did", time, gtype, pc), max_sub)
        write_record(f, np_tot.tobytes(), max_sub)
        for p in range(len(blocks)):
            for s in range(ntype):
                write_record(f, np.ascontiguousarray(blocks[p][s], dtype="<f8").tobytes(), max_sub)
