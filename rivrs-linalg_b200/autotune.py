"""Autotuner for the scheduling options of one sparsity pattern.

Two options only schedule the work: the large-front cutoff
(`large_front_threshold`: fronts at or above it take the whole GPU one after
another, the others are batched one CTA or warp per front) and, in the mixed
form without flushing, the Schur GEMM's tile width (`mixed_tile_cols`: 128, or
256 = two 128-column tiles sharing one W tile).  In the plain form neither
changes a result; the tile width changes none in the mixed form either, but
there the cutoff also decides which fronts take the tensor-core updates, so
the refined solution is checked by the caller as for any mixed factor.  Their
best values depend on the pattern (how many large fronts a wave holds, how
large).  `autotune` times
the candidates on the caller's own matrix with device-resident values (CUDA
events on the handle's stream, best of `reps` after one warm-up) and returns
the fastest; with `cache` set, results are kept in a JSON file keyed by the
pattern's fingerprint, the precision and the device, so a pattern is tuned once.

A third option changes the mixed factor's arithmetic: the window depth
(`mixed_window`, outer blocks of deferred updates).  Deeper windows move less
data and sum longer runs of products in FP32, so they are tried second, at the
best cutoff and tile width, only when the caller gives `step` (options ->
(seconds of one factor + solve to the caller's accuracy target, inertia)): a
deeper window is taken only if its whole step is faster and its inertia equals
`expect_inertia` (or, without it, the default window's).
There is no counterpart in the reference (its CPU path has no such options).
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
import os

import numpy as np

from .solver import FactorOptions, SparseLDLT

DEFAULT_THRESHOLDS = (1024, 2048, 4096)
DEFAULT_TILE_COLS = (128, 256)
DEFAULT_WINDOWS = (4, 8)


def fingerprint(solver: SparseLDLT) -> str:
    """Hash of the analysed structure (supernode ranges, patterns, parents)."""
    sym = solver.symbolic
    h = hashlib.sha256()
    for a in (sym.sup_begin, sym.sup_end, sym.sup_parent, np.diff(sym.pat_ptr)):
        h.update(np.ascontiguousarray(a, np.int64).tobytes())
    h.update(str(solver.system.n).encode())
    return h.hexdigest()[:24]


def candidates(base: FactorOptions, thresholds=DEFAULT_THRESHOLDS, tile_cols=DEFAULT_TILE_COLS) -> list:
    out = []
    tiles = tile_cols if (base.precision != "fp64" and base.mixed_flush == 0) else (base.mixed_tile_cols,)
    for t in thresholds:
        for c in tiles:
            out.append(dataclasses.replace(base, large_front_threshold=int(t), mixed_tile_cols=int(c)))
    return out


def _key(solver, base, device_name):
    return "|".join([fingerprint(solver), base.precision, base.mixed_operands, str(base.mixed_flush), device_name])


def _event_timer(solver: SparseLDLT, d_vals_ptr: int, d_scal_ptr: int | None, reps: int):
    """Seconds of one factorization with options o: one untimed run (sizes the
    arenas), then the best of `reps` runs timed by CUDA events on the handle's
    stream."""
    import torch

    def run(o: FactorOptions) -> float:
        solver._ensure_handle(o)
        st = torch.cuda.ExternalStream(solver.stream())
        solver.factor_device(d_vals_ptr, d_scal_ptr, o)
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            solver.factor_device(d_vals_ptr, d_scal_ptr, o)
            e1.record(st)
            e1.synchronize()
            t = e0.elapsed_time(e1) * 1e-3
            best = t if best is None else min(best, t)
        return best
    return run


def tune_window(best: FactorOptions, step, expect_inertia=None, windows=DEFAULT_WINDOWS):
    """(options, [(candidate as a dict, step seconds, inertia, accepted)]):
    the window depths tried at `best`'s other options; the default depth (the
    first of `windows`) is always acceptable, a deeper one only with the same
    inertia (expect_inertia, else the default depth's) and a faster step."""
    rows = []
    base_inertia = None
    for i, w in enumerate(windows):
        o = dataclasses.replace(best, mixed_window=int(w))
        sec, inertia = step(o)
        inertia = [int(v) for v in inertia]
        if i == 0:
            base_inertia = inertia
        ref = list(expect_inertia) if expect_inertia is not None else base_inertia
        rows.append(({"mixed_window": int(w)}, float(sec), inertia, i == 0 or inertia == [int(v) for v in ref]))
    pick = min((r for r in rows if r[3]), key=lambda r: r[1])
    return dataclasses.replace(best, **pick[0]), rows


def autotune(solver: SparseLDLT, d_vals_ptr: int | None, d_scal_ptr: int | None, base: FactorOptions, reps: int = 2,
             thresholds=DEFAULT_THRESHOLDS, tile_cols=DEFAULT_TILE_COLS, cache: str | None = None, timer=None,
             device_name: str | None = None, step=None, expect_inertia=None, windows=DEFAULT_WINDOWS):
    """(best options, [(candidate options as a dict, seconds)]) for factoring
    the values at d_vals_ptr (device) with the solver's pattern.  `timer`
    (options -> seconds) replaces the CUDA-event timing, `device_name` the
    current device's name in the cache key.  With `step` (mixed form without
    flushing), the window depth is tuned afterwards (tune_window); its rows
    follow the others in the table, with the step's seconds."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name()
    key = _key(solver, base, device_name)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            got = json.load(f).get(key)
        if got:
            return dataclasses.replace(base, **got["best"]), [(c, t) for c, t in got["table"]]
    run = timer or _event_timer(solver, d_vals_ptr, d_scal_ptr, reps)
    table = []
    for o in candidates(base, thresholds, tile_cols):
        table.append(({"large_front_threshold": o.large_front_threshold, "mixed_tile_cols": o.mixed_tile_cols},
                      float(run(o))))
    choice = min(table, key=lambda r: r[1])[0]
    if step is not None and base.precision != "fp64" and base.mixed_flush == 0 and len(windows) > 1:
        best, rows = tune_window(dataclasses.replace(base, **choice), step, expect_inertia, windows)
        choice = dict(choice, mixed_window=best.mixed_window)
        table += [(dict(c, step=True, inertia=inr, accepted=ok), sec) for c, sec, inr, ok in rows]
    if cache:
        data = {}
        if os.path.exists(cache):
            with open(cache) as f:
                data = json.load(f)
        data[key] = {"best": choice, "table": table}
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1)
        os.replace(tmp, cache)
    return dataclasses.replace(base, **choice), table
