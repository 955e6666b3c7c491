"""Many independent systems factored and solved together.

Systems are joined into block-diagonal unions (problems.block_diagonal), each
analysed once: a union's elimination forest has one tree per system, so the
level-set schedule of the numeric phase (factor_tree_levelset,
sparse/src/symmetric/numeric.rs:1957-2163) puts the fronts of every system
that sit at the same height into the same wave, and each wave's small and
medium fronts, across all the union's systems, go through the same batched
launches (one CTA or warp per front); large fronts take the whole GPU one
after another.  Each system's fronts, pivots and factors are exactly the ones
a separate factorization of that system with the same ordering and scaling
produces (its tree is untouched by the others).

A union holds every system's factor and contribution blocks at once, so the
systems are split, in order, into groups whose estimated device memory fits
a budget; `factor_solve` factors, solves and releases one group after the
other, `factor` + `solve` keep every group's factor (they must fit together).
Refactorization with new values reuses the analysis, the MC64 scaling and the
assembly maps of every group.  Right-hand sides of a group are solved
together, up to 8 per launch, systems with fewer columns padded with zeros.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as N
from . import problems
from .solver import AnalyzeOptions, FactorOptions, InvalidInput, OrderingStrategy, SparseLDLT

PT_1X1, PT_2X2 = 1, 2


def device_memory():
    """(free, total) bytes of the current device."""
    out = np.zeros(2, np.int64)
    st = N.lib().rvg_mem_info(out.ctypes.data_as(N.i64p))
    if st != 0:
        raise N.RvgError(N.lib().rvg_last_error().decode())
    return int(out[0]), int(out[1])


def memory_estimate(sym, outer_block: int = 256, nrhs: int = 8) -> tuple:
    """(factor bytes, workspace bytes) of one system's numeric phase, from its
    supernode structure and the delay-free level-set schedule: the factor is
    every front's m x k panel (8 bytes) plus indices and D; the workspace is
    the largest sum over a wave of the fronts' scratch plus the contribution
    blocks alive across waves (nfs^2 doubles each, from the child's wave to
    its parent's), and the solve vectors.  An upper bound of what the device
    arenas take (they are sized the same way)."""
    k = (sym.sup_end - sym.sup_begin).astype(np.int64)
    r = np.diff(sym.pat_ptr).astype(np.int64)
    m = k + r
    par = sym.sup_parent
    ns = k.size
    factor = float(np.sum(m * k)) * 8 * (1 + 1 / 16) + float(np.sum(m + k)) * 4 + float(np.sum(k)) * 17
    h = np.zeros(ns, np.int64)
    for s in range(ns):  # children precede their parents
        if par[s] >= 0 and h[par[s]] < h[s] + 1:
            h[par[s]] = h[s] + 1
    nh = int(h.max()) + 2 if ns else 1
    cb = (r.astype(np.float64) ** 2) * 8
    live = np.zeros(nh + 1)
    scr = np.zeros(nh + 1)
    for s in range(ns):
        if par[s] >= 0 and r[s] > 0:
            live[h[s]:h[par[s]] + 1] += cb[s]
        sc = (2 * 32 * m[s] + outer_block) * 8
        if m[s] >= 2048:
            sc = (m[s] * (2 * 32 + 4 * outer_block) + outer_block) * 8 + 2 * m[s] * 4 * outer_block * 8
        scr[h[s]] += max(sc, r[s] * k[s] * 8)
    work = float(np.max(live + scr)) + 2.0 * nrhs * float(np.sum(m)) * 8 + 16.0 * float(np.sum(m))
    return factor, work


@dataclass
class _Group:
    first: int           # first system of the group
    count: int
    union: problems.System
    solver: SparseLDLT
    sys_of_pos: np.ndarray  # elimination position -> system index within the group
    options: FactorOptions | None = None  # scheduling options tuned on this union (autotune_groups)


class BatchLDLT:
    def __init__(self, systems, scaling: bool = True, device_budget: int | None = None):
        """device_budget: bytes the groups may take (default: 80% of the free
        device memory now; 0 = a single union whatever its size)."""
        self.systems = list(systems)
        if not self.systems:
            raise InvalidInput("no systems")
        self.scaling = scaling
        self.offsets = np.cumsum([0] + [s.n for s in self.systems]).astype(np.int64)
        self.voffsets = np.cumsum([0] + [s.values.size for s in self.systems]).astype(np.int64)
        if device_budget is None:
            device_budget = int(0.8 * device_memory()[0])
        self.device_budget = device_budget
        est = [memory_estimate(SparseLDLT.analyze(s).symbolic) for s in self.systems] if device_budget else None
        self.estimates = est
        self.groups = []
        i = 0
        while i < len(self.systems):
            j = i + 1
            if device_budget:
                f, w = est[i]
                while j < len(self.systems) and (f + w + est[j][0] + est[j][1]) * 1.1 <= device_budget:
                    f, w = f + est[j][0], w + est[j][1]
                    j += 1
            else:
                j = len(self.systems)
            self.groups.append(self._make_group(i, j - i))
            i = j
        self._inertias = None

    def _make_group(self, first, count):
        union = problems.block_diagonal(self.systems[first:first + count], name=f"batch[{first}:{first + count}]")
        if self.scaling:
            solver = SparseLDLT.analyze_with_matrix(union, AnalyzeOptions(OrderingStrategy.MATCH_ORDER_METIS))
        else:
            solver = SparseLDLT.analyze(union)
        sop = np.searchsorted(union.meta["offsets"], solver.symbolic.perm_fwd, side="right") - 1
        return _Group(first, count, union, solver, sop)

    @property
    def n(self) -> int:
        return int(self.offsets[-1])

    # -- values and right-hand sides -------------------------------------------
    def values(self, per_system=None) -> np.ndarray:
        """The batch's values (the systems' value arrays in order) from one
        array per system (None: the systems' own values)."""
        if per_system is None:
            return np.concatenate([s.values for s in self.systems])
        if len(per_system) != len(self.systems):
            raise InvalidInput("one value array per system")
        for v, s in zip(per_system, self.systems):
            if np.asarray(v).size != s.values.size:
                raise InvalidInput("values do not match a system's pattern")
        return np.concatenate([np.asarray(v, dtype=np.float64) for v in per_system])

    def group_values(self, g: _Group, values: np.ndarray) -> np.ndarray:
        return values[self.voffsets[g.first]:self.voffsets[g.first + g.count]]

    def rhs_matrix(self, rhs_list, first: int = 0, count: int | None = None) -> np.ndarray:
        """Right-hand sides of systems [first, first + count) stacked (rows)
        and padded with zero columns to the widest (column-major)."""
        count = len(rhs_list) - first if count is None else count
        sub = rhs_list[first:first + count]
        cols = [1 if np.asarray(b).ndim == 1 else np.asarray(b).shape[1] for b in sub]
        lo0 = self.offsets[first]
        big = np.zeros((self.offsets[first + count] - lo0, max(cols)), order="F")
        for i, b in enumerate(sub):
            b = np.asarray(b, dtype=np.float64)
            lo, hi = self.offsets[first + i] - lo0, self.offsets[first + i + 1] - lo0
            if b.shape[0] != hi - lo:
                raise InvalidInput("right-hand side does not match its system")
            big[lo:hi, : cols[i]] = b if b.ndim == 2 else b[:, None]
        return big

    def split(self, x: np.ndarray, rhs_list, first: int = 0, count: int | None = None) -> list:
        count = len(rhs_list) - first if count is None else count
        out = []
        lo0 = self.offsets[first]
        for i in range(count):
            lo, hi = self.offsets[first + i] - lo0, self.offsets[first + i + 1] - lo0
            b = np.asarray(rhs_list[first + i])
            out.append(x[lo:hi, 0].copy() if b.ndim == 1 else np.asfortranarray(x[lo:hi, : b.shape[1]]))
        return out

    # -- numeric phase --------------------------------------------------------
    def factor(self, per_system=None, options: FactorOptions | None = None):
        """Factor every group and keep the factors (they must fit together;
        each group's workspace is released after its factorization when there
        are several groups)."""
        vals = self.values(per_system)
        inert = []
        for g in self.groups:
            g.solver.factor(self.group_values(g, vals), g.options if (options is None and g.options) else options)
            inert += self._group_inertias(g)
            if len(self.groups) > 1:
                g.solver.trim(workspace=True)
        self._inertias = inert

    refactor = factor

    def solve(self, rhs_list) -> list:
        """Solutions of every system (after factor()), shaped like its right-hand side."""
        if len(rhs_list) != len(self.systems):
            raise InvalidInput("one right-hand side per system")
        out = []
        for g in self.groups:
            big = self.rhs_matrix(rhs_list, g.first, g.count)
            x = g.solver.solve(big if big.shape[1] > 1 else big[:, 0])
            out += self.split(x.reshape(big.shape[0], -1, order="F"), rhs_list, g.first, g.count)
            if len(self.groups) > 1:
                g.solver.trim(workspace=True)
        return out

    def autotune_groups(self, d_values_ptr: int, d_scaling_ptrs=None, base: FactorOptions | None = None,
                        reps: int = 1, cache: str | None = None) -> list:
        """Tune the scheduling options of every group on its own union (the
        autotuner's candidates: large-front cutoff, and the tile width in the
        mixed form without flushing), the batch's values at d_values_ptr on
        the device (d_scaling_ptrs: one device scaling per group, or None).
        Each group keeps its choice in `options` (results are unchanged in
        the plain form) and releases its device memory afterwards.  Returns
        each group's table of (candidate, seconds)."""
        from . import autotune as at
        base = base or FactorOptions()
        tables = []
        for i, g in enumerate(self.groups):
            sp = None if d_scaling_ptrs is None else d_scaling_ptrs[i]
            tuned, table = at.autotune(g.solver, d_values_ptr + 8 * int(self.voffsets[g.first]), sp, base,
                                       reps=reps, cache=cache)
            g.options = tuned
            g.solver._ensure_handle(tuned)
            g.solver.trim(workspace=True, factor=True)
            tables.append(table)
        return tables

    def factor_solve(self, per_system, rhs_list, options: FactorOptions | None = None) -> list:
        """Factor and solve group by group, releasing each group's device
        memory (factor included) before the next: the batch only needs the
        largest group's memory."""
        if len(rhs_list) != len(self.systems):
            raise InvalidInput("one right-hand side per system")
        vals = self.values(per_system)
        out, inert = [], []
        for g in self.groups:
            g.solver.factor(self.group_values(g, vals), g.options if (options is None and g.options) else options)
            inert += self._group_inertias(g)
            big = self.rhs_matrix(rhs_list, g.first, g.count)
            x = g.solver.solve(big if big.shape[1] > 1 else big[:, 0])
            out += self.split(x.reshape(big.shape[0], -1, order="F"), rhs_list, g.first, g.count)
            g.solver.trim(workspace=True, factor=True)
        self._inertias = inert
        return out

    def _group_inertias(self, g: _Group) -> list:
        """(positive, negative, zero) per system of a factored group, from the
        pivots of its fronts (MixedDiagonal::compute_inertia,
        diagonal.rs:391-461)."""
        col, code, dd, do = g.solver.pivot_record()
        sysid = g.sys_of_pos[col]
        out = np.zeros((g.count, 3), np.int64)
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
        np.add.at(out[:, 2], s[z & (tr != 0)], 1)
        np.add.at(out[:, 2], s[z & (tr == 0)], 2)
        return [tuple(int(v) for v in r) for r in out]

    def inertias(self) -> list:
        """(positive, negative, zero) per system of the last factorization."""
        return self._inertias

    def system_record(self, i: int):
        """Pivot record (elimination position within the system, code, D
        diagonal, D off-diagonal) of system i (its group must hold its factor)."""
        g = next(g for g in self.groups if g.first <= i < g.first + g.count)
        col, code, dd, do = g.solver.pivot_record()
        sel = g.sys_of_pos[col] == i - g.first
        return col[sel] - col[sel].min(), code[sel], dd[sel], do[sel]

    def close(self):
        for g in self.groups:
            g.solver.close()
