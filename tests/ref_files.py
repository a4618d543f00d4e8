"""Readers of the files the reference writes and the library writes in the same layouts: the Tecplot
binary flow field (FieldIO, flowfield.plt, V112) and the statistics collections (SinglePointStat,
coll_*.bin).  Test helpers only."""
from pathlib import Path

import numpy as np


def _bytes(src):
    """A path or the file's bytes."""
    return bytes(src) if isinstance(src, (bytes, bytearray, memoryview)) else Path(src).read_bytes()


def read_plt(path):
    """Minimal reader of the V112 layout that ostc_write_plt and the reference's FieldIO write."""
    raw = _bytes(path)
    pos = 8
    assert raw[:8] == b"#!TDV112"

    def take(fmt, n=1):
        nonlocal pos
        v = np.frombuffer(raw, dtype=fmt, count=n, offset=pos)
        pos += v.nbytes
        return v

    def s():
        out = ""
        while True:
            c = int(take(np.int32)[0])
            if c == 0:
                return out
            out += chr(c)

    byte_order, file_type = (int(x) for x in take(np.int32, 2))
    assert (byte_order, file_type) == (1, 0)
    assert s() == "Solution file"
    nvar = int(take(np.int32)[0])
    names = [s() for _ in range(nvar)]
    zones = []
    marker = float(take(np.float32)[0])
    while marker == 299.0:
        name = s()
        parent, strand = (int(x) for x in take(np.int32, 2))
        t = float(take(np.float64)[0])
        color, ztype, loc, raw_nb, misc = (int(x) for x in take(np.int32, 5))
        dims = tuple(int(x) for x in take(np.int32, 3))
        aux = int(take(np.int32)[0])
        assert (parent, strand, color, ztype, loc, raw_nb, misc, aux) == (-1, -2, -1, 0, 0, 0, 0, 0)
        zones.append((name, t, dims))
        marker = float(take(np.float32)[0])
    assert marker == 357.0
    data = []
    for _, _, (nx, ny, nz) in zones:
        assert float(take(np.float32)[0]) == 299.0
        assert list(take(np.int32, nvar)) == [2] * nvar
        assert [int(x) for x in take(np.int32, 3)] == [0, 0, -1]
        mm = take(np.float64, 2 * nvar).reshape(nvar, 2)
        arr = take(np.float64, nvar * nx * ny * nz).reshape(nvar, nz, ny, nx)
        assert np.array_equal(mm[:, 0], arr.min(axis=(1, 2, 3))) and np.array_equal(mm[:, 1], arr.max(axis=(1, 2, 3)))
        data.append(arr)
    assert pos == len(raw)
    return names, zones, data


def read_stat_file(path):
    """The reference's coll_*.bin layout: int32 n_block, n_var, ngg; names as int32 characters each
    ended by 0; int32 counters[n_var]; per block int32 mx, my, mz and n_var planes of doubles."""
    raw = _bytes(path)
    pos = 0

    def ints(n):
        nonlocal pos
        v = np.frombuffer(raw, dtype=np.int32, count=n, offset=pos)
        pos += 4 * n
        return [int(x) for x in v]

    nb, nv, ngg = ints(3)
    names = []
    for _ in range(nv):
        name = ""
        while True:
            (c,) = ints(1)
            if c == 0:
                break
            name += chr(c)
        names.append(name)
    counters = ints(nv)
    blocks = []
    for _ in range(nb):
        mx, my, mz = ints(3)
        n = nv * (mx + 2 * ngg) * (my + 2 * ngg) * (mz + 2 * ngg)
        data = np.frombuffer(raw, dtype=np.float64, count=n, offset=pos)
        pos += 8 * n
        blocks.append(((mx, my, mz), data.reshape(nv, mz + 2 * ngg, my + 2 * ngg, mx + 2 * ngg)))
    assert pos == len(raw)
    return nb, ngg, names, counters, blocks
