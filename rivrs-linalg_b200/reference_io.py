"""Input files in the reference's formats: Matrix Market matrices and the
known-factorization JSON fixtures.

`load_mtx` reads `coordinate real symmetric` Matrix Market files as the
reference's `load_mtx` does (sparse/src/io/mtx.rs:27-172): any other header is
rejected, indices are 1-based and bounds-checked, explicit zeros are dropped
(they would add spurious edges to the ordering's graph), off-diagonal entries
are mirrored, and every malformed line is a ParseError naming its line.

The reference keeps, beside each hand-constructed test matrix, a companion
JSON file with an analytically known LDL^T factorization and loads it with
`load_reference` (sparse/src/io/reference.rs:70-117): a `permutation`
(0-indexed), the strict lower entries of unit-lower L (`l_entries`: row, col,
value), the block diagonal D (`d_blocks`: {"size": 1, "values": [d]} or
{"size": 2, "values": [[a, b], [c, d]]}, reference.rs:120-196) and the
`inertia`.  This module reads the same layout with the same checks (an entry
must have col < row, the permutation must hold every index once, a block must
have size 1 or 2 with values of that shape) and the same errors (IoError for
an unreadable file, ParseError otherwise), and rebuilds the matrix the
factorization describes, so fixtures can pin an oracle or a factorization.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

from .solver import IoError, ParseError

_MTX_HEADER = "%%matrixmarket matrix coordinate real symmetric"


def load_mtx(path, name: str | None = None):
    """A problems.System (both triangles stored) from a `coordinate real
    symmetric` Matrix Market file (mtx.rs:27-172)."""
    import scipy.sparse as sp

    from . import problems
    path = os.fspath(path)
    try:
        with open(path) as f:
            lines = f.read().splitlines()
    except OSError as e:
        raise IoError(path, str(e)) from None
    if not lines:
        raise ParseError(path, "empty file", 1)
    if not lines[0].lower().startswith(_MTX_HEADER):
        raise ParseError(path, "unsupported format: expected '%%MatrixMarket matrix coordinate real symmetric', "
                         f"got '{lines[0]}'", 1)
    i = 1
    while i < len(lines) and lines[i].startswith("%"):
        i += 1
    if i >= len(lines):
        raise ParseError(path, "missing size line")
    parts = lines[i].split()
    if len(parts) != 3:
        raise ParseError(path, f"size line must have 3 values (nrows ncols nnz), got {len(parts)}", i + 1)
    dims = []
    for what, tok in zip(("nrows", "ncols", "nnz"), parts):
        try:
            v = int(tok)
            if v < 0:
                raise ValueError
        except ValueError:
            raise ParseError(path, f"invalid {what}: '{tok}'", i + 1) from None
        dims.append(v)
    nrows, ncols, _ = dims
    rows, cols, vals = [], [], []
    for j in range(i + 1, len(lines)):
        line = lines[j].strip()
        if not line or line.startswith("%"):
            continue
        p = line.split()
        if len(p) != 3:
            raise ParseError(path, f"data line must have 3 values (row col val), got {len(p)}", j + 1)
        try:
            r = int(p[0])
        except ValueError:
            raise ParseError(path, f"invalid row index: '{p[0]}'", j + 1) from None
        try:
            c = int(p[1])
        except ValueError:
            raise ParseError(path, f"invalid col index: '{p[1]}'", j + 1) from None
        try:
            v = float(p[2])
        except ValueError:
            raise ParseError(path, f"invalid value: '{p[2]}'", j + 1) from None
        if r <= 0 or c <= 0:
            raise ParseError(path, "Matrix Market indices are 1-based; got 0", j + 1)
        r, c = r - 1, c - 1
        if r >= nrows or c >= ncols:
            raise ParseError(path, f"index ({r}, {c}) out of bounds for {nrows}x{ncols} matrix", j + 1)
        if v == 0.0:
            continue
        rows.append(r); cols.append(c); vals.append(v)
        if r != c:
            rows.append(c); cols.append(r); vals.append(v)
    a = sp.csc_matrix((np.array(vals, np.float64), (np.array(rows, np.int64), np.array(cols, np.int64))),
                      shape=(nrows, ncols))
    a.sum_duplicates()
    a.sort_indices()
    return problems.from_scipy(name or os.path.basename(path).rsplit(".", 1)[0], a)


@dataclass
class ReferenceFactorization:
    """ReferenceFactorization (reference.rs:45-60)."""
    matrix_name: str
    permutation: np.ndarray          # perm[new] = old
    l_rows: np.ndarray
    l_cols: np.ndarray
    l_values: np.ndarray
    d_blocks: list = field(default_factory=list)  # floats (1x1) or 2x2 arrays
    inertia: tuple = (0, 0, 0)       # (positive, negative, zero)
    notes: str = ""

    @property
    def n(self) -> int:
        return int(self.permutation.size)

    def l_dense(self) -> np.ndarray:
        L = np.eye(self.n)
        L[self.l_rows, self.l_cols] = self.l_values
        return L

    def d_dense(self) -> np.ndarray:
        D = np.zeros((self.n, self.n))
        i = 0
        for b in self.d_blocks:
            if np.ndim(b) == 0:
                D[i, i] = b
                i += 1
            else:
                D[i:i + 2, i:i + 2] = b
                i += 2
        return D

    def reconstruct(self) -> np.ndarray:
        """The symmetric matrix A with A[perm][:, perm] = L D L^T."""
        M = self.l_dense() @ self.d_dense() @ self.l_dense().T
        A = np.empty_like(M)
        p = self.permutation
        A[np.ix_(p, p)] = M
        return A

    def block_inertia(self) -> tuple:
        """(positive, negative, zero) eigenvalue counts of D (a 2x2 block by its
        determinant and trace, as MixedDiagonal::compute_inertia does)."""
        pos = neg = zero = 0
        for b in self.d_blocks:
            if np.ndim(b) == 0:
                pos += b > 0
                neg += b < 0
                zero += b == 0
            else:
                ev = np.linalg.eigvalsh(np.asarray(b, np.float64))
                pos += int(np.sum(ev > 0))
                neg += int(np.sum(ev < 0))
                zero += int(np.sum(ev == 0))
        return int(pos), int(neg), int(zero)


def _block(raw, i, path):
    if not isinstance(raw, dict):
        raise ParseError(path, "d_block must be an object")
    size = raw.get("size")
    if not isinstance(size, int) or isinstance(size, bool):
        raise ParseError(path, "d_block must have integer 'size' field")
    if "values" not in raw:
        raise ParseError(path, "d_block must have 'values' field")
    vals = raw["values"]
    if size == 1:
        if not isinstance(vals, list):
            raise ParseError(path, "1x1 d_block values must be an array")
        if len(vals) != 1:
            raise ParseError(path, f"1x1 d_block values must have exactly 1 element, got {len(vals)}")
        if not isinstance(vals[0], (int, float)) or isinstance(vals[0], bool):
            raise ParseError(path, "1x1 d_block value must be a number")
        return float(vals[0])
    if size == 2:
        if not isinstance(vals, list):
            raise ParseError(path, "2x2 d_block values must be an array")
        if len(vals) != 2:
            raise ParseError(path, f"2x2 d_block values must have exactly 2 rows, got {len(vals)}")
        out = np.zeros((2, 2))
        for r, row in enumerate(vals):
            if not isinstance(row, list):
                raise ParseError(path, f"2x2 d_block row {r} must be an array")
            if len(row) != 2:
                raise ParseError(path, f"2x2 d_block row {r} must have exactly 2 elements, got {len(row)}")
            for c, v in enumerate(row):
                if not isinstance(v, (int, float)) or isinstance(v, bool):
                    raise ParseError(path, f"2x2 d_block value at ({r}, {c}) must be a number")
                out[r, c] = v
        return out
    raise ParseError(path, f"d_block size must be 1 or 2, got {size}")


def parse_reference(obj, path: str = "<object>") -> ReferenceFactorization:
    """A ReferenceFactorization from the decoded JSON object, checked."""
    if not isinstance(obj, dict):
        raise ParseError(path, "expected a JSON object")
    for k in ("matrix_name", "permutation", "l_entries", "d_blocks", "inertia"):
        if k not in obj:
            raise ParseError(path, f"missing field `{k}`")
    try:
        perm = np.asarray(obj["permutation"], dtype=np.int64).ravel()
        ents = obj["l_entries"]
        rows = np.array([int(e["row"]) for e in ents], dtype=np.int64)
        cols = np.array([int(e["col"]) for e in ents], dtype=np.int64)
        vals = np.array([float(e["value"]) for e in ents], dtype=np.float64)
        inert = obj["inertia"]
        inertia = (int(inert["positive"]), int(inert["negative"]), int(inert["zero"]))
    except (TypeError, KeyError, ValueError) as e:
        raise ParseError(path, str(e)) from None
    if np.any(rows < 0) or np.any(cols < 0):
        raise ParseError(path, "negative index")
    for i in range(rows.size):  # reference.rs:87-98
        if cols[i] >= rows[i]:
            raise ParseError(path, f"l_entry[{i}] has col ({cols[i]}) >= row ({rows[i]}); must be strict lower triangle")
    n = perm.size  # validate_permutation (validate.rs), reference.rs:100-108
    seen = np.zeros(n, dtype=bool)
    for v in perm:
        if v < 0 or v >= n:
            raise ParseError(path, f"invalid permutation: index {v} out of range for n = {n}")
        if seen[v]:
            raise ParseError(path, f"invalid permutation: index {v} appears twice")
        seen[v] = True
    if rows.size and rows.max() >= n:
        raise ParseError(path, f"l_entry row {rows.max()} out of range for n = {n}")
    blocks = [_block(b, i, path) for i, b in enumerate(obj["d_blocks"])]
    return ReferenceFactorization(str(obj["matrix_name"]), perm, rows, cols, vals, blocks, inertia,
                                  str(obj.get("notes", "")))


def load_reference(path) -> ReferenceFactorization:
    """load_reference (reference.rs:70-117): IoError when the file cannot be
    read, ParseError on invalid JSON or inconsistent data."""
    path = os.fspath(path)
    try:
        with open(path) as f:
            content = f.read()
    except OSError as e:
        raise IoError(path, str(e)) from None
    try:
        obj = json.loads(content)
    except json.JSONDecodeError as e:
        raise ParseError(path, e.msg, e.lineno) from None
    return parse_reference(obj, path)
