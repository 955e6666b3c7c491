"""Learned per-front precision: which large fronts may take the mixed form.

The mixed form (precision="mixed") runs the Schur-complement updates of every
large front on the tensor cores with split FP64 operands; pivot tests, 2x2
inversions and storage stay FP64, and FP64 refinement (or GMRES-IR) wins the
accuracy back.  A front whose assembled matrix is badly conditioned loses more
in the mixed form, and refinement then needs more steps or stalls.  The
selector is a small perceptron (12 features, two hidden layers of 64, sigmoid
output; csrc/mlp.cuh) that predicts, from cheap features of each assembled
front computed on the device, whether the mixed form keeps that front's pivots
within bound; precision="learned" sends each large front to the mixed form or
to plain FP64 by that prediction.  A mixed front whose largest |D| entry grows
past growth_bound times its largest assembled entry makes the library factor
again in FP64, and `timed_solve` (factor, then solve to the tolerance)
refactors in FP64 when refinement stalls: the plain FP64 form is the
selector's fallback and arbiter.

Labels come from the solver itself (`label_fronts`): every matrix is factored
twice, all large fronts in FP64 and all in the mixed form, and a front is
"safe" when its mixed pivots match the FP64 ones (same 1x1/2x2/delay pattern)
and its D entries agree to a relative `tau`.  Training runs on the GPU through
the library's own forward/backward/Adam kernels (rvg_mlp_*), checked against
the float64 oracle in oracle/mlp_oracle.py.  None of this has a counterpart in
the reference crate.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from . import problems
from .solver import AnalyzeOptions, FactorOptions, OrderingStrategy, SparseLDLT

NFEAT = 12
FEATURE_NAMES = ("log2 m", "log2 k", "k/m", "log2(1+delayed in)", "delayed in/k", "log10 max|a|",
                 "log10 max|a_jj|/max|a|", "log10 min|a_jj|/max|a|", "log10 min column ratio",
                 "frac ratio<u", "frac negative diag", "frac zero diag")
# front table columns (rvg_front_features)
COL_S, COL_M, COL_K, COL_NE, COL_N1, COL_N2, COL_ROUTE, COL_PROB, COL_AMAX, COL_DMAX, COL_F0 = range(11)


def _check(st):
    N.check(st)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the selector's kernels need a GPU")
    return torch


class PrecisionSelector:
    """The network's parameters (float32, rvg_mlp_param_count() of them) and
    the decision threshold; training and inference run on the GPU."""

    def __init__(self, params: np.ndarray | None = None, seed: int = 0, threshold: float = 0.5,
                 growth_bound: float = 1e6):
        self.nparam = int(N.lib().rvg_mlp_param_count())
        self.ntrain = int(N.lib().rvg_mlp_trained_count())
        self.threshold = threshold
        self.growth_bound = growth_bound
        if params is None:
            rng = np.random.default_rng(seed)
            h = 64
            p = np.zeros(self.nparam, np.float32)
            o = 0
            p[o:o + h * NFEAT] = rng.normal(0, np.sqrt(2.0 / NFEAT), h * NFEAT); o += h * NFEAT
            o += h  # b1
            p[o:o + h * h] = rng.normal(0, np.sqrt(2.0 / h), h * h); o += h * h
            o += h  # b2
            p[o:o + h] = rng.normal(0, np.sqrt(1.0 / h), h); o += h
            o += 1  # b3
            p[o:o + NFEAT] = 0.0
            p[o + NFEAT:o + 2 * NFEAT] = 1.0
            params = p
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        if self.params.size != self.nparam:
            raise ValueError("selector parameters have the wrong length")

    # normalisation (mean, standard deviation per feature), not trained
    def fit_normalisation(self, X: np.ndarray):
        X = np.asarray(X, np.float64)
        self.params[self.ntrain:self.ntrain + NFEAT] = X.mean(0)
        self.params[self.ntrain + NFEAT:] = np.maximum(X.std(0), 1e-3)

    def train(self, X, y, weights=None, steps: int = 1500, lr: float = 3e-3, weight_decay: float = 1e-4,
              log_every: int = 100) -> list:
        """Full-batch Adam on the GPU kernels; returns [(step, loss)]."""
        torch = _torch()
        L = N.lib()
        X = np.ascontiguousarray(X, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        n = y.size
        if weights is None:  # balance the classes
            pos = max(float(y.sum()), 1.0)
            neg = max(float(n - y.sum()), 1.0)
            weights = np.where(y > 0.5, 0.5 * n / pos, 0.5 * n / neg)
        w = np.ascontiguousarray(weights, np.float32)
        dev = "cuda"
        dP = torch.from_numpy(self.params.copy()).to(dev)
        dX, dY, dW = (torch.from_numpy(a).to(dev) for a in (X, y, w))
        dG = torch.zeros(self.ntrain, dtype=torch.float32, device=dev)
        dM, dV = torch.zeros_like(dG), torch.zeros_like(dG)
        dL = torch.zeros(1, dtype=torch.float32, device=dev)
        work = torch.empty(int(L.rvg_mlp_work_floats(n)), dtype=torch.float32, device=dev)
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        hist = []
        norm = float(w.sum())
        for t in range(1, steps + 1):
            _check(L.rvg_mlp_grad(C.c_void_p(dP.data_ptr()), C.c_void_p(dX.data_ptr()), C.c_void_p(dY.data_ptr()),
                                  C.c_void_p(dW.data_ptr()), n, norm, C.c_void_p(dG.data_ptr()),
                                  C.c_void_p(dL.data_ptr()), C.c_void_p(work.data_ptr()), work.numel(), st))
            if t == 1 or t % log_every == 0 or t == steps:
                hist.append((t, float(dL.item())))
            _check(L.rvg_mlp_adam(C.c_void_p(dP.data_ptr()), C.c_void_p(dG.data_ptr()), C.c_void_p(dM.data_ptr()),
                                  C.c_void_p(dV.data_ptr()), t, lr, 0.9, 0.999, 1e-8, weight_decay, st))
        torch.cuda.synchronize()
        self.params = dP.cpu().numpy()
        return hist

    def predict_proba(self, X) -> np.ndarray:
        torch = _torch()
        X = np.ascontiguousarray(X, np.float32)
        if X.shape[0] == 0:
            return np.zeros(0, np.float32)
        dP = torch.from_numpy(self.params).to("cuda")
        dX = torch.from_numpy(X).to("cuda")
        out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        _check(N.lib().rvg_mlp_forward(C.c_void_p(dP.data_ptr()), C.c_void_p(dX.data_ptr()), X.shape[0],
                                       C.c_void_p(out.data_ptr()), st))
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def save(self, path):
        np.savez(path, params=self.params, threshold=self.threshold, growth_bound=self.growth_bound)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z["params"], threshold=float(z["threshold"]), growth_bound=float(z["growth_bound"]))


class _Forced:
    """A stand-in selector that sends every large front one way."""

    def __init__(self, nparam, ntrain, mixed: bool):
        self.params = np.zeros(nparam, np.float32)
        self.params[ntrain + NFEAT:] = 1.0
        self.threshold = -1.0 if mixed else 2.0
        self.growth_bound = 1e300


def c5_family(count: int, seed: int, grid_lo: int, grid_hi: int) -> list:
    """Generated matrices for labels: alternately a shifted 7-point Laplacian
    with the shift at a U[1%, 20%] fraction of the spectrum and a KKT whose H
    regularisation is diag(U[0, 10^U[-8, -2]]), on grids uniform in
    [grid_lo, grid_hi]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        g = int(rng.integers(grid_lo, grid_hi + 1))
        if i % 2 == 0:
            out.append(problems.shifted_laplacian(g, float(rng.uniform(0.01, 0.20))))
        else:
            kg = max(4, int(round(g * 0.8)))
            for attempt in range(8):
                try:
                    out.append(problems.kkt(kg, seed=int(rng.integers(1 << 30)),
                                            reg_hi=float(10.0 ** rng.uniform(-8, -2))))
                    break
                except RuntimeError:
                    continue
    return out


def _front_slices(solver):
    """Per supernode: (first position in the pivot record, eliminated count)."""
    fi = solver.front_info()
    ne = fi[:, 2]
    start = np.concatenate([[0], np.cumsum(ne)[:-1]])
    return start, ne


@dataclass
class Labelled:
    X: np.ndarray          # features (fronts x 12), from the FP64 run
    y: np.ndarray          # 1 = the mixed form is safe for the front
    err: np.ndarray        # relative D difference (inf when the pivot pattern differs)
    m: np.ndarray          # front orders
    system: list = field(default_factory=list)  # index of the matrix of each front


def label_fronts(system, tau: float = 1e-3, opts: FactorOptions | None = None, scaling: bool = True):
    """Factor `system` with every large front in FP64 and then in the mixed
    form; per large front its features (FP64 run), the relative difference of
    its D entries and the label err <= tau with an identical pivot pattern."""
    base = opts or FactorOptions(large_front_threshold=256, mixed_flush=0, mixed_operands="bf16")
    lo = FactorOptions(**{**base.__dict__, "precision": "learned"})
    solver = (SparseLDLT.analyze_with_matrix(system, AnalyzeOptions(OrderingStrategy.MATCH_ORDER_METIS))
              if scaling else SparseLDLT.analyze(system))
    nparam, ntrain = int(N.lib().rvg_mlp_param_count()), int(N.lib().rvg_mlp_trained_count())
    runs = []
    for mixed in (False, True):
        solver.set_selector(_Forced(nparam, ntrain, mixed))
        solver.factor(None, lo)
        rows = solver.front_features()
        col, code, dd, do = solver.pivot_record()
        start, ne = _front_slices(solver)
        runs.append((rows, code.copy(), dd.copy(), do.copy(), start, ne))
    solver.close()
    (r64, c64, d64, o64, s64, n64), (rmx, cmx, dmx, omx, smx, nmx) = runs
    mx_row = {int(r[COL_S]): r for r in rmx}
    X, y, err, m = [], [], [], []
    for r in r64:
        s = int(r[COL_S])
        if s not in mx_row:
            continue
        e = np.inf
        if n64[s] == nmx[s]:
            a0, b0 = s64[s], smx[s]
            k = n64[s]
            if np.array_equal(c64[a0:a0 + k], cmx[b0:b0 + k]):
                ref = np.concatenate([d64[a0:a0 + k], o64[a0:a0 + k]])
                got = np.concatenate([dmx[b0:b0 + k], omx[b0:b0 + k]])
                scale = max(np.max(np.abs(ref)) if ref.size else 0.0, 1e-300)
                e = float(np.max(np.abs(got - ref)) / scale) if ref.size else 0.0
        X.append(r[COL_F0:COL_F0 + NFEAT])
        err.append(e)
        y.append(1.0 if e <= tau else 0.0)
        m.append(r[COL_M])
    return (np.array(X, np.float64).reshape(-1, NFEAT), np.array(y), np.array(err), np.array(m))


def label_family(systems, tau: float = 1e-3, opts: FactorOptions | None = None, scaling: bool = True) -> Labelled:
    Xs, ys, es, ms, ids = [], [], [], [], []
    for i, s in enumerate(systems):
        X, y, e, m = label_fronts(s, tau, opts, scaling)
        Xs.append(X); ys.append(y); es.append(e); ms.append(m); ids += [i] * len(y)
    return Labelled(np.concatenate(Xs) if Xs else np.zeros((0, NFEAT)), np.concatenate(ys) if ys else np.zeros(0),
                    np.concatenate(es) if es else np.zeros(0), np.concatenate(ms) if ms else np.zeros(0), ids)


def sample_weights(data: Labelled, cost_power: float = 0.5) -> np.ndarray:
    """Training weights: the two classes balanced, and each front weighted by
    (m k / mean m k) ** cost_power, since the large fronts carry the time."""
    y = data.y
    n = max(y.size, 1)
    pos, neg = max(float(y.sum()), 1.0), max(float(n - y.sum()), 1.0)
    w = np.where(y > 0.5, 0.5 * n / pos, 0.5 * n / neg)
    k = 2.0 ** data.X[:, 1] if data.X.size else np.zeros(0)
    cost = data.m * k
    if cost_power and cost.size:
        w = w * (cost / cost.mean()) ** cost_power
    return w


def misprediction(selector: PrecisionSelector, data: Labelled) -> dict:
    """Rates on labelled fronts: unsafe fronts sent to the mixed form (the
    costly mistake), safe fronts kept in FP64 (lost speed), and overall."""
    p = selector.predict_proba(data.X) if data.y.size else np.zeros(0)
    return misprediction_of(p, selector.threshold, data.y)


def misprediction_of(p: np.ndarray, threshold: float, y: np.ndarray) -> dict:
    """misprediction() from the probabilities themselves."""
    route = np.asarray(p) >= threshold
    safe = np.asarray(y) > 0.5
    n = max(safe.size, 1)
    return dict(fronts=int(safe.size), safe=int(safe.sum()), routed_mixed=int(route.sum()),
                unsafe_sent_mixed=int((route & ~safe).sum()), safe_kept_fp64=int((~route & safe).sum()),
                rate=float(((route & ~safe) | (~route & safe)).sum() / n))


def timed_solve(solver, system, opts: FactorOptions, b, tol=1e-14, warmup: int = 0):
    """Factor + solve to `tol` (refinement escalating to GMRES-IR; FP64
    refactorization when that stalls), timed on the host with the device
    synchronised, after `warmup` untimed runs (the first run with new
    options also creates the handle and sizes its arenas); returns a dict."""
    import torch
    for _ in range(warmup):
        solver.factor(None, opts)
        solver.solve_auto(b, tol=tol)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    solver.factor(None, opts)
    fp64_rerun = False
    x, its, err, how = solver.solve_auto(b, tol=tol)
    if not err <= tol and opts.precision != "fp64":
        fp64_rerun = True
        solver.factor(None, FactorOptions(**{**opts.__dict__, "precision": "fp64"}))
        x, its2, err, how = solver.solve_auto(b, tol=tol)
        its += its2
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    pr = solver.profile()
    out = dict(s=t, factor_gpu_s=pr["factor_ms"] * 1e-3, bwd=float(problems.backward_error(system, x, b)),
               solves_after_first=int(its), method=how, refactored_fp64=fp64_rerun)
    if opts.precision == "learned":
        out.update(solver.selector_stats())
    return out
