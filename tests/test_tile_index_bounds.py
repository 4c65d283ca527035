"""Index arithmetic of the 2D tile launches, checked on the CPU.

The large-level tile kernels (mg_fused.cu: k_relax_tile2d_w on FP32 levels,
k_relax_tile2d_x4 on FP64 levels) read a 64 x 64 staged region per tile and,
in the first launch of a level, the bilinear prolongation of the level below
(prolong_row / prolong_cell).  This restates their index formulas with the
library's level geometry (mg_host.c make_geom: P = roundup(xo + n + 1, align),
n + 2 rows) and checks, for every tile and thread of the levels 512^2 to
4096^2, that each element they address lies inside its level array and, for
the coarse level, inside its real cells or its one-cell ghost ring (the only
values the coarse relaxation writes)."""
import numpy as np
import pytest

W = 64


def geom(n, xo, align):
    P = (xo + n + 1 + align - 1) // align * align
    return {"n": n, "xo": xo, "P": P, "size": (n + 2) * P}


def cidx(g, i, j):
    return (i + 1) * g["P"] + g["xo"] + j


# (storage, tile size TS, cells per thread K, xo, row alignment)
CONFIGS = [("f32", 48, 8, 8, 32), ("f32", 32, 8, 8, 32), ("f64", 48, 4, 4, 16)]


def tiles(n, ts):
    h = (W - ts) // 2
    nt = (n + ts - 1) // ts
    b = np.arange(nt)
    by, bx = np.meshgrid(b, b, indexing="ij")
    return by.ravel() * ts - h, bx.ravel() * ts - h


@pytest.mark.parametrize("st,ts,k,xo,align", CONFIGS)
@pytest.mark.parametrize("depth", [9, 10, 11, 12])
def test_fused_prolongation_reads_stay_in_the_coarse_level(st, ts, k, xo, align, depth):
    n = 1 << depth
    gf, gc = geom(n, xo, align), geom(n // 2, xo, align)
    nc = gc["n"]
    i0, j0 = tiles(n, ts)
    inner = (i0 >= 0) & (i0 + W <= n) & (j0 >= 0) & (j0 + W <= n)
    p = np.arange(W)[:, None]                    # staged row of a thread
    q0 = k * np.arange(W // k)[None, :]          # first of its k columns
    # interior tiles: prolong_row over columns jb .. jb + k - 1 of row gi
    for a, b in zip(i0[inner], j0[inner]):
        gi, jb = a + p, b + q0
        assert (jb % 2 == 0).all()               # the row's first column is even
        ci, cx = gi >> 1, np.where(gi & 1, 1, -1)
        cb = (jb >> 1) - 1
        for row in (ci, ci + cx):
            assert row.min() >= -1 and row.max() <= nc
            first, last = cidx(gc, row, cb), cidx(gc, row, cb + k // 2 + 1)
            assert cb.min() >= -1 and (cb + k // 2 + 1).max() <= nc
            assert first.min() >= 0 and last.max() < gc["size"]
    # boundary tiles: prolong_cell at every real cell (non-periodic: real
    # cells only; periodic images map into the same range)
    for a, b in zip(i0[~inner], j0[~inner]):
        gi, gj = a + p, b + np.arange(W)[None, :]
        real = (gi >= 0) & (gi < n) & (gj >= 0) & (gj < n)
        ri, rj = np.broadcast_to(gi, real.shape)[real], np.broadcast_to(gj, real.shape)[real]
        ci, cj = ri >> 1, rj >> 1
        for di in (0, 1):
            for dj in (0, 1):
                ii = ci + di * np.where(ri & 1, 1, -1)
                jj = cj + dj * np.where(rj & 1, 1, -1)
                assert ii.min() >= -1 and ii.max() <= nc and jj.min() >= -1 and jj.max() <= nc
                e = cidx(gc, ii, jj)
                assert e.min() >= 0 and e.max() < gc["size"]


@pytest.mark.parametrize("st,ts,k,xo,align", CONFIGS)
@pytest.mark.parametrize("depth", [9, 10, 11, 12])
def test_interior_tile_loads_stay_in_the_level(st, ts, k, xo, align, depth):
    """The interior-tile loads of the same kernels: k cells of res and of the
    iterate, alpha_x on the rows of faces gi and gi + 1, alpha_y on k + 1
    faces, all vector loads aligned to 16 bytes."""
    n = 1 << depth
    g = geom(n, xo, align)
    es = 4 if st == "f32" else 8
    i0, j0 = tiles(n, ts)
    inner = (i0 >= 0) & (i0 + W <= n) & (j0 >= 0) & (j0 + W <= n)
    p = np.arange(W)[:, None]
    q0 = k * np.arange(W // k)[None, :]
    for a, b in zip(i0[inner], j0[inner]):
        gi, jb = a + p, b + q0
        first = cidx(g, gi, jb)
        assert (first * es % 16 == 0).all()      # quad loads
        assert first.min() >= 0
        assert cidx(g, gi + 1, jb + k - 1).max() < g["size"]      # alpha_x, row gi + 1
        assert (cidx(g, gi, jb + k) <= cidx(g, gi, 0) + g["P"] - g["xo"] - 1).all()  # alpha_y, face jb + k in the row
