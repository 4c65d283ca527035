"""Host logic of the block decomposition (no device needed):
MPI_Dims_create and MPI_Cart_shift as the library computes them."""
import pytest

from basilisk_b200.shard import dims_create, neighbours


@pytest.mark.parametrize("n,dim,want", [
    (1, 2, (1, 1)), (2, 2, (2, 1)), (4, 2, (2, 2)), (6, 2, (3, 2)), (7, 2, (7, 1)),
    (8, 2, (4, 2)), (16, 2, (4, 4)), (8, 3, (2, 2, 2)), (12, 3, (3, 2, 2)),
    (24, 3, (4, 3, 2)), (64, 3, (4, 4, 4)), (2, 1, (2,))])
def test_dims_create(n, dim, want):
    """MPI_Dims_create (n, dim) with all dims free: balanced, non-increasing."""
    assert dims_create(n, dim) == want


@pytest.mark.parametrize("dims,periodic", [((2, 2), ()), ((4, 2), (0,)), ((3, 2), (0, 1)),
                                            ((2, 2, 2), (0, 1, 2)), ((4, 1), (1,)),
                                            ((3, 3, 2), (2,))])
def test_neighbours_are_mutual(dims, periodic):
    """Every side that faces a block is faced back by that block's opposite
    side (each exchange has its matching message), box sides are exactly
    the domain's non-periodic ends, and a single-block periodic direction
    has no neighbours (the block's own periodic images)."""
    dim = len(dims)
    nb = 1
    for d in dims:
        nb *= d
    stride = [1] * dim
    for e in range(dim - 2, -1, -1):
        stride[e] = stride[e + 1] * dims[e + 1]
    for b in range(nb):
        nbr = neighbours(dim, dims, periodic, b)
        c = [(b // stride[e]) % dims[e] for e in range(dim)]
        for e in range(dim):
            for hi in (0, 1):
                s = 2 * e + (0 if hi else 1)
                edge = c[e] == (dims[e] - 1 if hi else 0)
                if dims[e] == 1 or (edge and e not in periodic):
                    assert nbr[s] == -1, (b, s, nbr)
                    continue
                o = nbr[s]
                co = [(o // stride[k]) % dims[k] for k in range(dim)]
                assert co[e] == (c[e] + (1 if hi else -1)) % dims[e]
                assert all(co[k] == c[k] for k in range(dim) if k != e)
                back = neighbours(dim, dims, periodic, o)
                assert back[2 * e + (1 if hi else 0)] == b
