"""The grid nested-dissection ordering: a permutation, identical to the
box-by-box construction it replaces, with separators after both halves."""
import numpy as np
import pytest


def reference_nd(dims, leaf=8):
    """Box by box: each box's nodes in C order, in dissection order."""
    nx, ny, nz = dims
    out = []

    def emit(x0, x1, y0, y1, z0, z1):
        i, j, k = np.meshgrid(np.arange(x0, x1), np.arange(y0, y1), np.arange(z0, z1), indexing="ij")
        out.append((i * ny * nz + j * nz + k).ravel())
    stack = [((0, nx, 0, ny, 0, nz), None)]
    while stack:
        box, sep = stack.pop()
        if sep is not None:
            emit(*sep)
            continue
        x0, x1, y0, y1, z0, z1 = box
        sx, sy, sz = x1 - x0, y1 - y0, z1 - z0
        if sx <= 0 or sy <= 0 or sz <= 0:
            continue
        if sx * sy * sz <= leaf or max(sx, sy, sz) < 3:
            emit(*box)
            continue
        if sx >= sy and sx >= sz:
            mid = x0 + sx // 2
            a, b, s = (x0, mid, y0, y1, z0, z1), (mid + 1, x1, y0, y1, z0, z1), (mid, mid + 1, y0, y1, z0, z1)
        elif sy >= sz:
            mid = y0 + sy // 2
            a, b, s = (x0, x1, y0, mid, z0, z1), (x0, x1, mid + 1, y1, z0, z1), (x0, x1, mid, mid + 1, z0, z1)
        else:
            mid = z0 + sz // 2
            a, b, s = (x0, x1, y0, y1, z0, mid), (x0, x1, y0, y1, mid + 1, z1), (x0, x1, y0, y1, mid, mid + 1)
        stack.append((None, s))
        stack.append((b, None))
        stack.append((a, None))
    return np.concatenate(out).astype(np.int64)


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 1), (5, 5, 5), (7, 3, 9), (16, 16, 16), (17, 4, 29), (30, 30, 30),
                                  (27, 27, 27)])
@pytest.mark.parametrize("leaf", [1, 8, 64])
def test_matches_box_by_box(rv, dims, leaf):
    got = rv.ordering.nested_dissection_grid(dims, leaf)
    assert np.array_equal(got, reference_nd(dims, leaf))
    assert np.array_equal(np.sort(got), np.arange(np.prod(dims)))


def test_large_grid_is_a_permutation_with_separator_last(rv):
    n = 60
    o = rv.ordering.nested_dissection_grid((n, n, n))
    assert np.array_equal(np.sort(o), np.arange(n ** 3))
    # the top separator (the plane x = 30) is numbered last
    last = o[-n * n:]
    assert np.all(last // (n * n) == n // 2)
    assert np.array_equal(o, reference_nd((n, n, n)))
