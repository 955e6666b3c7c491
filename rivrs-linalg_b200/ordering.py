"""Fill-reducing orderings supplied to the analysis (UserSupplied semantics,
sparse/src/symmetric/solver.rs:51-52).

METIS (the reference's default, reached through the metis-sys crate at
sparse/src/ordering/metis.rs:559-600) is not available to this build, so:

* grid problems use exact geometric nested dissection: a box is split along
  its longest side by a one-node-thick plane, which separates both the
  7-point and the 27-point stencil; halves first, separator last;
* the KKT systems order H by the same dissection of its grid and put the
  constraint rows last (their Schur complement -J H^-1 J^T is dense and
  negative definite, so the last front takes 1x1 pivots);
* other matrices fall back to reverse Cuthill-McKee or the natural order.

All functions return ``order`` with ``order[new] = old`` (int64).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def dissection_boxes(dims, leaf: int = 8) -> np.ndarray:
    """The boxes of the geometric nested dissection of an nx*ny*nz grid in the
    order their nodes are numbered (rows x0, x1, y0, y1, z0, z1): a box is
    split along its longest side (x, then y, then z on ties) at the middle
    plane; its first half, then its second half, then the plane; a box of at
    most `leaf` nodes or with every side shorter than 3 is a leaf."""
    nx, ny, nz = dims
    boxes = []
    # explicit stack of (box, is_separator)
    stack = [((0, nx, 0, ny, 0, nz), False)]
    while stack:
        box, is_sep = stack.pop()
        x0, x1, y0, y1, z0, z1 = box
        sx, sy, sz = x1 - x0, y1 - y0, z1 - z0
        if sx <= 0 or sy <= 0 or sz <= 0:
            continue
        if is_sep or sx * sy * sz <= leaf or max(sx, sy, sz) < 3:
            boxes.append(box)
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
        # LIFO: push in reverse of the order wanted (a, b, separator)
        stack.append((s, True))
        stack.append((b, False))
        stack.append((a, False))
    return np.array(boxes, dtype=np.int64).reshape(-1, 6)


def nested_dissection_grid(dims, leaf: int = 8) -> np.ndarray:
    """Geometric nested dissection of an nx*ny*nz grid (linear index
    i*ny*nz + j*nz + k, i.e. C order of (i, j, k)); within a box its nodes
    are numbered in C order too.  The boxes come from dissection_boxes; their
    nodes are expanded for all boxes at once."""
    nx, ny, nz = dims
    b = dissection_boxes(dims, leaf)
    sx, sy, sz = b[:, 1] - b[:, 0], b[:, 3] - b[:, 2], b[:, 5] - b[:, 4]
    size = sx * sy * sz
    n = int(size.sum())
    assert n == nx * ny * nz
    box = np.repeat(np.arange(b.shape[0]), size)
    start = np.concatenate([[0], np.cumsum(size)[:-1]])
    q = np.arange(n, dtype=np.int64) - start[box]
    plane = (sy * sz)[box]
    i = b[box, 0] + q // plane
    r = q % plane
    j = b[box, 2] + r // sz[box]
    k = b[box, 4] + r % sz[box]
    return (i * ny * nz + j * nz + k).astype(np.int64)


def kkt_order(sysm, leaf: int = 8) -> np.ndarray:
    """H by nested dissection of its grid, then the constraint rows."""
    h = nested_dissection_grid(sysm.grid, leaf)
    return np.concatenate([h, np.arange(sysm.n_h, sysm.n, dtype=np.int64)])


def rcm_order(sysm) -> np.ndarray:
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    a = sysm.to_scipy()
    return np.asarray(reverse_cuthill_mckee(a.tocsr(), symmetric_mode=True), dtype=np.int64)


def natural_order(n: int) -> np.ndarray:
    return np.arange(n, dtype=np.int64)


def default_order(sysm) -> np.ndarray:
    if "parts" in sysm.meta:  # block-diagonal union: each block's own order, blocks in sequence
        offs = sysm.meta["offsets"]
        return np.concatenate([default_order(p) + o for p, o in zip(sysm.meta["parts"], offs[:-1])])
    if sysm.grid is not None and sysm.n_h == 0:
        return nested_dissection_grid(sysm.grid)
    if sysm.grid is not None and sysm.n_h > 0:
        return kkt_order(sysm)
    if sysm.n <= 2:
        return natural_order(sysm.n)
    return rcm_order(sysm)


def mc64(sysm):
    """MC64 maximum-product matching and symmetric scaling (mc64_matching,
    sparse/src/ordering/matching.rs:121-248), computed on the host by the
    library (rvg_mc64).  Returns (matching, scaling, matched) in the system's
    original index order: matching[i] is the column matched to row i,
    scaling[i] the symmetric scaling factor, matched the number of matched
    rows (n for structurally nonsingular matrices)."""
    from . import _native as N
    n = int(sysm.n)
    colptr = N.as_i64(sysm.colptr)
    rowidx = N.as_i64(sysm.rowidx)
    vals = N.as_f64(sysm.values)
    matching = np.zeros(max(n, 1), np.int64)
    scaling = np.zeros(max(n, 1), np.float64)
    matched = C.c_int64(0)
    st = N.lib().rvg_mc64(n, N.ptr(colptr, N.i64p), N.ptr(rowidx, N.i64p), N.ptr(vals, N.dp),
                          N.ptr(matching, N.i64p), N.ptr(scaling, N.dp), C.byref(matched))
    if st != 0:
        raise N.RvgError(st, N.lib().rvg_last_error().decode())
    return matching[:n], scaling[:n], int(matched.value)
