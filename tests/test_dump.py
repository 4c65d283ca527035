"""dump () / restore () (output.h:1043-1400): the oracle's independent writer
against a hand-assembled file, and the library's bmg_dump / bmg_restore
against the oracle's writer and reader, byte for byte.

The reference's own tests of this pair (test/pdump.c writing restore.dump,
test/restore.c, restore-tree.c and restore-multigrid.c reading it back and
asserting s[] == sin(x)*cos(y) on every leaf) are mirrored by
test_pdump_restore_* below: the same depth-6 grids, origin (-0.5, -0.5), the
same refinement condition, the same assertion."""
import math
import os
import struct

import numpy as np
import pytest

from oracle import dumpfile

DEPTH = 6


def pdump_cond(level, x, y):
    """test/pdump.c: refine (level < depth - 2 || level <= depth*(1. -
    sqrt(x*x + y*y + z*z))) with z = 0."""
    return level < DEPTH - 2 or level <= DEPTH * (1. - math.sqrt(x * x + y * y))


def sincos(x, y):
    return np.vectorize(lambda a, b: math.sin(a) * math.cos(b))(x, y)


def centers(level, X0=-0.5, Y0=-0.5, L0=1.0):
    n = 1 << level
    c = (np.arange(n) + 0.5) * (L0 * (1.0 / n))
    return np.meshgrid(c + X0, c + Y0, indexing="ij")


def test_known_answer_bytes(tmp_path):
    """A depth-1 uniform grid assembled field by field from the struct
    definitions of output.h: header, names, origin, then the root (not a
    leaf, subtree of 5 cells) and its four children in foreach_cell order."""
    lv = [np.array([[7.0]]), np.array([[1.0, 2.0], [3.0, 4.0]])]
    p = tmp_path / "k.dump"
    dumpfile.write_dump(p, 2, 1, [("s", lv)], t=0.25, i=3, origin=(-0.5, -0.5, -0.5), L0=2.0)
    want = struct.pack("<d", 0.25) + struct.pack("<q", 2) + struct.pack("<4i", 3, 1, 1, 170901)
    want += struct.pack("<3d", 0, 0, 0)
    want += struct.pack("<I", 4) + b"size" + struct.pack("<I", 1) + b"s"
    want += struct.pack("<4d", -0.5, -0.5, -0.5, 2.0)
    want += struct.pack("<I2d", 0, 5.0, 7.0)
    for v in (1.0, 2.0, 3.0, 4.0):          # (0,0) (0,1) (1,0) (1,1)
        want += struct.pack("<I2d", 2, 1.0, v)
    assert p.read_bytes() == want
    d = dumpfile.read_dump(p, 2)
    assert (d["t"], d["i"], d["depth"], d["npe"], d["names"]) == (0.25, 3, 1, 1, ["size", "s"])
    assert d["origin"] == (-0.5, -0.5, -0.5) and d["L0"] == 2.0


def test_oracle_tree_round_trip(tmp_path):
    """pdump.c's tree on the tree oracle: the file holds its active cells
    with the subtree sizes, and reads back to the same leaves and values."""
    from oracle import tree as otree
    t = otree.Tree(DEPTH, origin=(-0.5, -0.5))
    t.refine(pdump_cond)
    leaf = [(t.flags(l) & otree.LEAF) != 0 for l in range(t.depth + 1)]
    active = [(t.flags(l) & otree.ACTIVE) != 0 for l in range(t.depth + 1)]
    vals = [np.where(leaf[l], sincos(*centers(l)), 0.0) for l in range(t.depth + 1)]
    p = tmp_path / "tree.dump"
    dumpfile.write_dump(p, 2, t.depth, [("s", vals)], leaf=leaf, origin=(-0.5, -0.5, -0.5))
    d = dumpfile.read_dump(p, 2)
    assert len(d["cells"]) == sum(int(a.sum()) for a in active)
    assert d["cells"][0][3][0] == len(d["cells"])        # root subtree = every cell
    v, lf = dumpfile.level_arrays(d, 2, "s")
    for l in range(t.depth + 1):
        np.testing.assert_array_equal(lf[l], leaf[l])
        np.testing.assert_array_equal(v[l][leaf[l]], vals[l][leaf[l]])
    assert sum(int(m.sum()) for m in lf) == t.leaves


def test_legacy_format(tmp_path):
    p = tmp_path / "old.dump"
    lv = [np.array([[1.5]]), np.arange(4.0).reshape(2, 2)]
    dumpfile.write_dump(p, 2, 1, [("a", lv)], version=dumpfile.LEGACY)
    d = dumpfile.read_dump(p, 2, legacy_names=["a"])
    assert d["version"] == 161020 and d["names"] == ["size", "a"]
    assert [c[3][1] for c in d["cells"]] == [1.5, 0.0, 1.0, 2.0, 3.0]


# ---------------------------------------------------------------- GPU --

def _uniform_levels(dim, depth, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((1 << l,) * dim) for l in range(depth + 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("dim,depth", [(2, 5), (3, 3)])
def test_dump_uniform_bytes(tmp_path, dim, depth):
    """bmg_dump of a uniform grid writes the oracle writer's file byte for
    byte (all levels, foreach_cell order, subtree sizes)."""
    import basilisk_b200 as bmg
    g = bmg.Grid(dim, depth, L0=2.0, origin=(-1.0, 0.5, 0.25)[:dim])
    a, b = g.scalar(), g.scalar()
    la, lb = _uniform_levels(dim, depth, 1), _uniform_levels(dim, depth, 2)
    for l in range(depth + 1):
        a.set(la[l], level=l)
        b.set(lb[l], level=l)
    p = tmp_path / "g.dump"
    g.dump(str(p), {"a": a, "b": b}, t=1.5, i=42)
    q = tmp_path / "o.dump"
    o = (-1.0, 0.5, 0.25) if dim == 3 else (-1.0, 0.5, 0.0)
    dumpfile.write_dump(q, dim, depth, [("a", la), ("b", lb)], t=1.5, i=42, origin=o, L0=2.0)
    assert p.read_bytes() == q.read_bytes()
    assert not os.path.exists(str(p) + "~")
    g.close()


@pytest.mark.gpu
def test_pdump_restore_multigrid(tmp_path):
    """test/pdump-multigrid.c then test/restore-multigrid.c: a depth-6
    uniform grid with s = sin(x)*cos(y), dumped, restored into a fresh grid
    whose origin the file sets."""
    import basilisk_b200 as bmg
    g = bmg.Grid(2, DEPTH, origin=(-0.5, -0.5))
    s = g.scalar(sincos(*centers(DEPTH)))
    p = tmp_path / "restore.dump"
    g.dump(str(p), {"s": s})
    g.close()
    h = bmg.Grid(2, DEPTH)
    s2 = h.scalar()
    t, i = h.restore(str(p), {"s": s2})
    assert (t, i) == (0.0, 0) and h.origin[:2] == (-0.5, -0.5)
    np.testing.assert_array_equal(s2.get(), sincos(*centers(DEPTH, *h.origin[:2])))
    h.close()


@pytest.mark.gpu
def test_pdump_restore_tree(tmp_path):
    """test/pdump.c (tree) then test/restore-tree.c: the quadtree of
    pdump.c's condition with s = sin(x)*cos(y) on its leaves; the file
    matches the oracle's writer on the tree oracle byte for byte, and a
    fresh tree grid restored from it has the same cells and leaf values."""
    import basilisk_b200 as bmg
    from oracle import tree as otree
    g = bmg.TreeGrid(DEPTH, origin=(-0.5, -0.5))
    g.refine(pdump_cond)
    s = g.scalar()
    depth = g.tree_depth
    leaf = [g.leaf_mask(l) for l in range(depth + 1)]
    vals = [np.where(leaf[l], sincos(*centers(l)), 0.0) for l in range(depth + 1)]
    for l in range(depth + 1):
        s.set(vals[l], level=l)
    p = tmp_path / "restore-tree.dump"
    g.dump(str(p), {"s": s}, t=0.5, i=7)
    t = otree.Tree(DEPTH, origin=(-0.5, -0.5))
    t.refine(pdump_cond)
    oleaf = [(t.flags(l) & otree.LEAF) != 0 for l in range(t.depth + 1)]
    q = tmp_path / "oracle.dump"
    dumpfile.write_dump(q, 2, t.depth, [("s", vals)], leaf=oleaf, t=0.5, i=7,
                        origin=(-0.5, -0.5, 0.0))
    assert p.read_bytes() == q.read_bytes()
    h = bmg.TreeGrid(DEPTH)
    h.refine(lambda l, x, y: l < 2)          # replaced by the file's tree
    s2 = h.scalar()
    assert h.restore(str(p), {"s": s2}) == (0.5, 7)
    assert h.tree_depth == depth and h.leaves == g.leaves
    for l in range(depth + 1):
        np.testing.assert_array_equal(h.flags(l), g.flags(l))
        got = s2.get(level=l)
        np.testing.assert_array_equal(got[leaf[l]], sincos(*h.centers(l))[leaf[l]])
    g.close()
    h.close()


@pytest.mark.gpu
def test_restore_oracle_files(tmp_path):
    """Files written by the oracle: columns matched by name in any order,
    unknown columns skipped, the legacy unnamed format, a uniform file read
    by a tree grid (a full tree), and a tree file read by a uniform grid."""
    import basilisk_b200 as bmg
    depth = 4
    la, lb, lc = (_uniform_levels(2, depth, k) for k in (3, 4, 5))
    p = tmp_path / "abc.dump"
    dumpfile.write_dump(p, 2, depth, [("a", la), ("b", lb), ("c", lc)], t=2.0, i=9)
    g = bmg.Grid(2, depth)
    fc, fa = g.scalar(), g.scalar()
    assert g.restore(str(p), [("c", fc), ("a", fa)]) == (2.0, 9)
    for l in range(depth + 1):
        np.testing.assert_array_equal(fc.get(level=l), lc[l])
        np.testing.assert_array_equal(fa.get(level=l), la[l])
    q = tmp_path / "legacy.dump"
    dumpfile.write_dump(q, 2, depth, [("x", lb)], version=dumpfile.LEGACY)
    fx = g.scalar()
    g.restore(str(q), [("x", fx)])
    np.testing.assert_array_equal(fx.get(), lb[depth])
    with pytest.raises(RuntimeError):          # legacy: the list must match the columns
        g.restore(str(q), [("x", fx), ("y", fa)])
    g.close()
    h = bmg.TreeGrid(depth + 1)
    fb = h.scalar()
    h.restore(str(p), {"b": fb})
    assert h.tree_depth == depth and h.leaves == 1 << (2 * depth)
    for l in range(depth + 1):
        np.testing.assert_array_equal(fb.get(level=l), lb[l])
    h.close()
    # a tree file into a uniform grid: the grid becomes that tree
    from oracle import tree as otree
    t = otree.Tree(depth)
    t.refine(lambda l, x, y: l < 2 or (l < depth and x < 0.3 and y > 0.6))
    leaf = [(t.flags(l) & otree.LEAF) != 0 for l in range(t.depth + 1)]
    r = tmp_path / "tree.dump"
    dumpfile.write_dump(r, 2, t.depth, [("a", la)], leaf=leaf)
    u = bmg.Grid(2, depth)
    fa = u.scalar()
    u.restore(str(r), {"a": fa})
    for l in range(t.depth + 1):
        np.testing.assert_array_equal(bmg.TreeGrid.flags(u, l) & 3, t.flags(l) & 3)
        m = (t.flags(l) & otree.ACTIVE) != 0
        np.testing.assert_array_equal(fa.get(level=l)[m], la[l][m])
    u.close()


@pytest.mark.gpu
def test_restore_errors(tmp_path):
    import basilisk_b200 as bmg
    g = bmg.Grid(2, 4)
    s = g.scalar()
    with pytest.raises(RuntimeError):
        g.restore(str(tmp_path / "missing.dump"), {"s": s})
    p = tmp_path / "d3.dump"
    dumpfile.write_dump(p, 2, 3, [("s", _uniform_levels(2, 3, 0))])
    with pytest.raises(RuntimeError):          # a uniform file of another depth
        g.restore(str(p), {"s": s})
    q = tmp_path / "short.dump"
    q.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(RuntimeError):          # truncated
        g.restore(str(q), {"s": s})
    g.close()
