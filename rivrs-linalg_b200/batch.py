"""Many independent systems factored and solved together.

The systems become the diagonal blocks of one block-diagonal system
(problems.block_diagonal), analysed once: the union's elimination forest has
one tree per system, so the level-set schedule of the numeric phase
(factor_tree_levelset, sparse/src/symmetric/numeric.rs:1957-2163) puts the
fronts of every system that sit at the same height into the same wave, and
each wave's small and medium fronts, across all systems, go through the same
batched launches (one CTA or warp per front); large fronts take the whole GPU
one after another.  Each system's fronts, pivots and factors are exactly the
ones a separate factorization of that system with the same ordering and
scaling produces (its tree is untouched by the others).

Refactorization with new values (`factor(values)` again) reuses the
analysis, the MC64 scaling, the assembly maps and every device buffer of the
handle.  Right-hand sides of all systems are solved together, up to 8 per
launch, systems with fewer columns padded with zeros.
"""
from __future__ import annotations

import numpy as np

from . import problems
from .solver import AnalyzeOptions, FactorOptions, InvalidInput, OrderingStrategy, SparseLDLT

PT_1X1, PT_2X2 = 1, 2


class BatchLDLT:
    def __init__(self, systems, scaling: bool = True):
        self.systems = list(systems)
        if not self.systems:
            raise InvalidInput("no systems")
        self.union = problems.block_diagonal(self.systems)
        self.offsets = self.union.meta["offsets"]
        if scaling:
            self.solver = SparseLDLT.analyze_with_matrix(self.union, AnalyzeOptions(OrderingStrategy.MATCH_ORDER_METIS))
        else:
            self.solver = SparseLDLT.analyze(self.union)
        # elimination position -> system
        self._sys_of_pos = np.searchsorted(self.offsets, self.solver.symbolic.perm_fwd, side="right") - 1

    @property
    def n(self) -> int:
        return int(self.union.n)

    def values(self, per_system=None) -> np.ndarray:
        """The union's values from one value array per system (None: the
        systems' own values)."""
        if per_system is None:
            return self.union.values
        if len(per_system) != len(self.systems):
            raise InvalidInput("one value array per system")
        for v, s in zip(per_system, self.systems):
            if np.asarray(v).size != s.values.size:
                raise InvalidInput("values do not match a system's pattern")
        return np.concatenate([np.asarray(v, dtype=np.float64) for v in per_system])

    def factor(self, per_system=None, options: FactorOptions | None = None):
        self.solver.factor(self.values(per_system), options)

    refactor = factor

    def factor_device(self, d_values_ptr: int, d_scaling_ptr: int | None, options: FactorOptions | None = None):
        """Factor from union values already on the device (`values()` layout)."""
        self.solver.factor_device(d_values_ptr, d_scaling_ptr, options)

    def rhs_matrix(self, rhs_list) -> np.ndarray:
        """The union's right-hand sides (n x max columns, column-major),
        systems with fewer columns padded with zeros."""
        cols = [1 if np.asarray(b).ndim == 1 else np.asarray(b).shape[1] for b in rhs_list]
        big = np.zeros((self.n, max(cols)), order="F")
        for i, b in enumerate(rhs_list):
            b = np.asarray(b, dtype=np.float64)
            lo, hi = self.offsets[i], self.offsets[i + 1]
            if b.shape[0] != hi - lo:
                raise InvalidInput("right-hand side does not match its system")
            big[lo:hi, : cols[i]] = b if b.ndim == 2 else b[:, None]
        return big

    def split(self, x: np.ndarray, rhs_list) -> list:
        out = []
        for i, b in enumerate(rhs_list):
            lo, hi = self.offsets[i], self.offsets[i + 1]
            b = np.asarray(b)
            out.append(x[lo:hi, 0].copy() if b.ndim == 1 else np.asfortranarray(x[lo:hi, : b.shape[1]]))
        return out

    def solve(self, rhs_list) -> list:
        """Solutions of every system, shaped like its right-hand side."""
        if len(rhs_list) != len(self.systems):
            raise InvalidInput("one right-hand side per system")
        big = self.rhs_matrix(rhs_list)
        x = self.solver.solve(big if big.shape[1] > 1 else big[:, 0])
        return self.split(x.reshape(self.n, -1, order="F"), rhs_list)

    def inertias(self) -> list:
        """(positive, negative, zero) per system, from the pivots of its fronts
        (MixedDiagonal::compute_inertia, diagonal.rs:391-461)."""
        col, code, dd, do = self.solver.pivot_record()
        sysid = self._sys_of_pos[col]
        out = np.zeros((len(self.systems), 3), np.int64)
        one = code == PT_1X1
        np.add.at(out[:, 0], sysid[one & (dd > 0)], 1)
        np.add.at(out[:, 1], sysid[one & (dd < 0)], 1)
        np.add.at(out[:, 2], sysid[one & (dd == 0)], 1)
        first = np.nonzero(code == PT_2X2)[0]
        a, b, c = dd[first], do[first], dd[first + 1]
        det = a * c - b * b
        tr = a + c
        s = sysid[first]
        np.add.at(out[:, 0], s[(det > 0) & (tr > 0)], 2)
        np.add.at(out[:, 1], s[(det > 0) & ~(tr > 0)], 2)
        np.add.at(out[:, 0], s[det < 0], 1)
        np.add.at(out[:, 1], s[det < 0], 1)
        z = det == 0
        np.add.at(out[:, 0], s[z & (tr > 0)], 1)
        np.add.at(out[:, 1], s[z & (tr < 0)], 1)
        np.add.at(out[:, 2], s[z & (tr > 0)], 1)
        np.add.at(out[:, 2], s[z & (tr < 0)], 1)
        np.add.at(out[:, 2], s[z & (tr == 0)], 2)
        return [tuple(int(v) for v in r) for r in out]

    def close(self):
        self.solver.close()
