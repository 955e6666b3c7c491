"""Trains the per-front precision selector on generated matrices.

    python rivrs-linalg_b200/train_selector.py --count 200 --grid 14 30 --out selector.npz

Labels come from factoring every matrix twice on the GPU (all large fronts in
FP64, then all in the mixed form; selector.label_fronts); the matrices are
split by matrix into training and validation sets, the network is trained by
the library's own CUDA kernels (full-batch Adam), and the validation
misprediction rates are printed with the saved parameters' path.
"""
import argparse
import json
import os
import sys
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=200)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--grid", type=int, nargs=2, default=(14, 30))
    ap.add_argument("--tau", type=float, default=1e-4)
    ap.add_argument("--large-threshold", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--val-fraction", type=float, default=0.2)
    ap.add_argument("--out", default="selector.npz")
    ap.add_argument("--save-data", default=None, help="also save the labelled fronts (npz)")
    ap.add_argument("--cost-weight", type=float, default=0.5,
                    help="sample weight grows as (m k / mean m k) ** this (large fronts dominate the time)")
    a = ap.parse_args(argv)
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    import __graft_entry__ as entry
    rv = entry.load_package()
    S = rv.selector
    t0 = time.perf_counter()
    fam = S.c5_family(a.count, a.seed, a.grid[0], a.grid[1])
    opts = rv.FactorOptions(large_front_threshold=a.large_threshold, mixed_flush=0, mixed_operands="bf16")
    data = S.label_family(fam, a.tau, opts)
    t_label = time.perf_counter() - t0
    if a.save_data:
        np.savez(a.save_data, X=data.X, y=data.y, err=data.err, m=data.m, system=np.asarray(data.system))
    ids = np.asarray(data.system)
    nval = max(1, int(round(a.val_fraction * len(fam))))
    val_sys = set(range(len(fam) - nval, len(fam)))
    val = np.isin(ids, list(val_sys))
    tr = S.Labelled(data.X[~val], data.y[~val], data.err[~val], data.m[~val], list(ids[~val]))
    va = S.Labelled(data.X[val], data.y[val], data.err[val], data.m[val], list(ids[val]))
    sel = S.PrecisionSelector(seed=a.seed)
    sel.fit_normalisation(tr.X)
    t1 = time.perf_counter()
    hist = sel.train(tr.X, tr.y, weights=S.sample_weights(tr, a.cost_weight), steps=a.steps, lr=a.lr)
    t_train = time.perf_counter() - t1
    sel.save(a.out)
    rep = dict(matrices=len(fam), fronts=int(data.y.size), safe_fraction=float(data.y.mean()) if data.y.size else None,
               tau=a.tau, label_s=t_label, train_s=t_train, loss_first=hist[0][1], loss_last=hist[-1][1],
               train=S.misprediction(sel, tr), validation=S.misprediction(sel, va), out=a.out)
    print(json.dumps(rep))
    return sel, rep


if __name__ == "__main__":
    main()
