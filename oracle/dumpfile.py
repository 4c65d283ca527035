"""Basilisk snapshot files (``dump ()`` / ``restore ()``, output.h:1043-1400),
restated in plain Python.

TEST INFRASTRUCTURE ONLY: an independent writer and reader of the
reference's binary format, used by ``tests/`` to check the library's
``bmg_dump`` / ``bmg_restore`` byte for byte.  The product never imports it.

Format (single process, dump_version 170901):
  header   struct DumpHeader {double t; long len; int i, depth, npe, version;
           coord n;}, 56 bytes, native byte order (output.h:1050-1058)
  names    len of them: unsigned length + characters, "size" first
           (output.h:1070-1086, 1113-1117)
  origin   double o[4] = {X0, Y0, Z0, L0} (output.h:1087-1091)
  cells    foreach_cell () order (grid/foreach_cell.h:86-112: depth first,
           children with the x index slowest, z fastest), not below leaves:
           unsigned flags (leaf = 2), then len doubles: the subtree's cell
           count (subtree_size (size, false), multigrid-common.h:422-440)
           and the fields (output.h:1122-1135)
The older version 161020 has no names section (output.h:1265-1273).
"""
import struct

import numpy as np

VERSION = 170901
LEGACY = 161020
LEAF = 2
HEADER = struct.Struct("=dq4i3d")       # 56 bytes (long is 64-bit)


def _children(dim, i, j, k):
    for c in range(1 << dim):
        ci = 2 * i + ((c >> (dim - 1)) & 1)
        cj = 2 * j + ((c >> (dim - 2)) & 1) if dim > 1 else 0
        ck = 2 * k + (c & 1) if dim > 2 else 0
        yield ci, cj, ck


def _index(dim, i, j, k):
    return (i,) if dim == 1 else (i, j) if dim == 2 else (i, j, k)


def write_dump(path, dim, depth, fields, leaf=None, t=0.0, i=0, origin=(0.0, 0.0, 0.0),
               L0=1.0, version=VERSION):
    """fields: list of (name, [level arrays of shape (2**l,)*dim]).  leaf:
    None for a uniform grid (the leaves are level depth), else per-level
    boolean masks of the leaves of a tree (cells below leaves are not
    written)."""
    def is_leaf(l, ci, cj, ck):
        return l == depth if leaf is None else bool(leaf[l][_index(dim, ci, cj, ck)])

    size = {}

    def subtree(l, ci, cj, ck):
        if is_leaf(l, ci, cj, ck) or l == depth:
            s = 1.0
        else:
            s = 1.0 + sum(subtree(l + 1, *c) for c in _children(dim, ci, cj, ck))
        size[(l, ci, cj, ck)] = s
        return s

    subtree(0, 0, 0, 0)
    out = bytearray()
    out += HEADER.pack(t, len(fields) + 1, i, depth, 1, version, 0.0, 0.0, 0.0)
    if version != LEGACY:
        for name in ["size"] + [n for n, _ in fields]:
            b = name.encode()
            out += struct.pack("=I", len(b)) + b
    out += struct.pack("=4d", origin[0], origin[1], origin[2], L0)

    def emit(l, ci, cj, ck):
        lf = is_leaf(l, ci, cj, ck)
        out.extend(struct.pack("=I", LEAF if lf else 0))
        vals = [size[(l, ci, cj, ck)]] + [float(v[l][_index(dim, ci, cj, ck)]) for _, v in fields]
        out.extend(struct.pack("=%dd" % len(vals), *vals))
        if not lf:
            for c in _children(dim, ci, cj, ck):
                emit(l + 1, *c)

    emit(0, 0, 0, 0)
    with open(path, "wb") as fp:
        fp.write(bytes(out))


def read_dump(path, dim, legacy_names=None):
    """Parses a dump: returns dict(t, i, depth, npe, version, names, origin,
    L0, cells) where cells is a list of (level, (i, j, k), leaf, values)."""
    with open(path, "rb") as fp:
        data = fp.read()
    t, ln, it, depth, npe, version, _, _, _ = HEADER.unpack_from(data, 0)
    pos = HEADER.size
    if version == LEGACY:
        names = ["size"] + list(legacy_names or ["f%d" % q for q in range(ln - 1)])
    else:
        names = []
        for _ in range(ln):
            (n,) = struct.unpack_from("=I", data, pos)
            names.append(data[pos + 4:pos + 4 + n].decode())
            pos += 4 + n
    o = struct.unpack_from("=4d", data, pos)
    pos += 32
    cells = []

    def parse(l, ci, cj, ck):
        nonlocal pos
        (flags,) = struct.unpack_from("=I", data, pos)
        vals = struct.unpack_from("=%dd" % ln, data, pos + 4)
        pos += 4 + 8 * ln
        lf = bool(flags & LEAF)
        cells.append((l, (ci, cj, ck), lf, vals))
        if not lf:
            for c in _children(dim, ci, cj, ck):
                parse(l + 1, *c)

    parse(0, 0, 0, 0)
    if pos != len(data):
        raise ValueError("trailing bytes in %s: %d of %d read" % (path, pos, len(data)))
    return dict(t=t, i=it, depth=depth, npe=npe, version=version, names=names,
                origin=o[:3], L0=o[3], cells=cells)


def level_arrays(dump, dim, name):
    """The values of one named column, per level (NaN where the file has no
    cell), and per-level leaf masks."""
    col = dump["names"].index(name)
    depth = dump["depth"]
    vals = [np.full((1 << l,) * dim, np.nan) for l in range(depth + 1)]
    leaf = [np.zeros((1 << l,) * dim, dtype=bool) for l in range(depth + 1)]
    for l, (ci, cj, ck), lf, v in dump["cells"]:
        vals[l][_index(dim, ci, cj, ck)] = v[col]
        leaf[l][_index(dim, ci, cj, ck)] = lf
    return vals, leaf
