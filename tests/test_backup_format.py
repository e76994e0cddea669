"""The backup file format checker (oracle/fortran_records.py) against scipy's Fortran reader
for single-subrecord files, and its multi-subrecord layout."""
import struct

import numpy as np
from scipy.io import FortranFile

from oracle import fortran_records as FR


def test_records_match_scipy(tmp_path):
    p = tmp_path / "a.bak"
    rng = np.random.default_rng(1)
    blocks = [[rng.random((5, 6)), rng.random((0, 6))], [rng.random((3, 6)), rng.random((7, 6))]]
    FR.write_backup(str(p), 1.25e-6, 3, 0.75, blocks)
    f = FortranFile(str(p), "r", header_dtype="<i4")
    head = f.read_record("<f8", "<i4", "<f8")
    assert head[0][0] == 1.25e-6 and head[1][0] == 3 and head[2][0] == 0.75
    assert list(f.read_ints("<i4")) == [5, 0, 3, 7]
    for pr in range(2):
        for s in range(2):
            a = f.read_reals("<f8").reshape(-1, 6)
            assert np.array_equal(a, blocks[pr][s])
    f.close()
    t, g, pc, np_tot, parts = FR.read_backup(str(p), 2)
    assert (t, g, pc) == (1.25e-6, 3, 0.75) and np_tot.tolist() == [[5, 0], [3, 7]]
    assert np.array_equal(parts[1][1], blocks[1][1])


def test_subrecord_layout(tmp_path):
    p = tmp_path / "b.bin"
    data = bytes(range(256)) * 3          # 768 bytes in subrecords of 300
    with open(p, "wb") as f:
        FR.write_record(f, data, max_sub=300)
    raw = p.read_bytes()
    # subrecords 300, 300, 168: leading -300, -300, 168; trailing 300, -300, -168
    marks = []
    pos = 0
    for k in (300, 300, 168):
        lead, = struct.unpack("<i", raw[pos:pos + 4]); pos += 4 + k
        tail, = struct.unpack("<i", raw[pos:pos + 4]); pos += 4
        marks.append((lead, tail))
    assert marks == [(-300, 300), (-300, -300), (168, -168)] and pos == len(raw)
    with open(p, "rb") as f:
        assert FR.read_record(f) == data
