#!/usr/bin/env python
"""Benchmark of the B200 numeric phase (factor + solve) on one synthetic system.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config C] [--impl b200|reference]

A step is one numeric factorization plus the solve of the whole system to a
scaled backward error of 1e-14 (the metric: factor+solve time to that
accuracy).  The default workload is the saddle-point KKT system
[[H, J^T], [J, 0]] with H the 27-point Laplacian of a 60^3 grid plus
diag(U[0,1e-2]) and J 54,000 x 216,000 with 4 N(0,1) entries per row
(n = 270,000), MC64-scaled, one right-hand side b ~ N(0,1).  Forms timed:
plain FP64; the mixed form (Schur updates on the tcgen05 tensor cores) with
TF32 operand parts at the flush depths of --mixed-flush, followed by FP64
iterative refinement; with BF16 parts at the depths of --bf16-flush,
followed by GMRES-IR.  `value` is the fastest form that reaches 1e-14.

* `value`  seconds per step with the matrix values and the RHS already in HBM
           (CUDA events on the handle's stream, max over ranks; the library's
           per-launch profiling events off).
* `e2e`    the same step through the public API with host buffers (values and
           RHS copied in, x copied out).
* `roofline` the chosen form's Schur-complement GEMM (from one extra profiled
           step): executed flops / its event-timed device time, against a
           GEMM peak of the same arithmetic (cuBLAS measured in the run, or
           the measured-peaks file for BF16).
* `hbm_bound_parts` the solve and the assembly against the measured HBM
           copy bandwidth.
* `cpu_baseline` the CPU restatement of the reference numeric phase
           (oracle/, blocked, OpenMP on every host core) on a bounded part
           of THIS workload's factorization (about 20 s), scaled to the
           whole by flops.
`--impl reference` runs that CPU restatement alone (oracle libraries only, no
GPU library) through ONE complete factor + solve of the workload, timed in
`--steps` consecutive slices of the factorization; its value is the sum of
the slices.
`--config batch64` times the many-systems workload instead (64 systems,
grouped unions; see run_batch).  Multi-GPU runs are independent replicas
(the single-system path does not shard): each rank factors its own copy, no
collective in the data path.
"""

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (builder, description)
    "kkt60": ("kkt", 60, "kkt27_60^3: H 27-pt 60^3 + diag U[0,1e-2], J 54000x216000 (4/row), n=270000"),
    "kkt36": ("kkt", 36, "kkt27_36^3 (the KKT family at n=58320; profiling case)"),
    "kkt48": ("kkt", 48, "kkt27_48^3 (the KKT family at n=138240; profiling case)"),
    "lap16": ("lap", 16, "laplace7_16^3 shifted to 10% negative, n=4096"),
    "lap100": ("lap", 100, "laplace7_100^3 shifted to 5% negative, n=1000000"),
    "batch64": ("batch", 64, "64 systems, n log-uniform in [5e3, 2e5] (seed 1), half shifted 7-pt Laplacians, "
                "half KKT, 1-32 RHS each; then 20 refactorizations"),
    "learned": ("learned", 0, "per-front precision selector: trained on 200 generated matrices (shift U[1%,20%], "
                "KKT regularisation 10^U[-8,-2], grids 20^3-60^3), evaluated on held-out matrices: laplace7_100^3 "
                "at 5% negative (n=1e6) and a kkt27_60^3 with a held-out seed (n=270000)"),
}
SELECTOR = os.path.join(ROOT, "rivrs-linalg_b200", "data", "selector_bf16.npz")
METRIC = "factor+solve time to bwd err 1e-14, chosen form vs plain FP64 on 1 B200"


def analyze(rv, s):
    """MatchOrderMetis analysis (the reference's default ordering strategy): MC64
    matching + symmetric scaling on the host, this project's nested-dissection
    order.  Returns the solver and the host time of the analysis in ms."""
    t0 = time.perf_counter()
    solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
    return solver, (time.perf_counter() - t0) * 1e3


def build_system(rv, cfg):
    kind, g, _ = CONFIGS[cfg]
    if kind == "kkt":
        s = rv.problems.kkt(g, seed=0)
        b = rv.problems.rhs_normal(s.n, seed=0)
    else:
        s = rv.problems.shifted_laplacian(g, 0.10 if g < 100 else 0.05)
        b = rv.problems.rhs_uniform(s.n, seed=0)
    return s, b


def dense_flops(sym):
    """Delay-free factor + Schur flops of the supernode structure (2 per multiply-add)."""
    k = (sym.sup_end - sym.sup_begin).astype(np.float64)
    r = np.diff(sym.pat_ptr).astype(np.float64)
    # panel: sum_j [(m-j-1) + (m-j-1)(m-j)] over the k eliminated columns (m = k + r)
    m = k + r
    j = k
    s1 = j * (m - 1) - j * (j - 1) / 2  # sum of (m-j-1)
    # sum_{t=0}^{k-1} (m-t-1)(m-t) = sum_{u=m-k}^{m-1} u(u+1)
    def sq(n):
        return n * (n + 1) * (2 * n + 1) / 6

    def lin(n):
        return n * (n + 1) / 2
    s2 = (sq(m - 1) + lin(m - 1)) - (sq(m - k - 1) + lin(m - k - 1))
    return float(np.sum(s1 + s2))


def cpu_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def cpu_analyze(rv, orc, s):
    """The analysis for a CPU-only run: the project's ordering and the
    library's host symbolic analysis + MC64 through the oracle's analysis
    library (no GPU library loaded)."""
    return orc.analyze(s, rv.ordering.default_order(s), mc64=True)


def cpu_sample(rv, orc, s, b, budget_s=20.0):
    """The CPU restatement of the reference's numeric phase on THIS workload
    for a bounded time: the factorization runs in slices of 2% of its
    delay-free flops until budget_s have passed; the time is scaled to the
    whole factorization by flops (a bounded sample, not a full run)."""
    sym, sc = cpu_analyze(rv, orc, s)
    threads = cpu_threads()
    f = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=threads, sliced=True)
    tot = f.total_flops()
    t, frac, ended = 0.0, 0.0, False
    while t < budget_s and not ended:
        frac = min(1.0, frac + 0.02)
        t0 = time.perf_counter()
        ended = f.advance(tot * frac if frac < 1.0 else 1e300)
        t += time.perf_counter() - t0
    done = orc.lib().orc_session_done(f.session) if not ended else tot
    f.close()
    orc.release_cache()
    value = t * tot / max(done, 1.0)
    return dict(value=value, unit="s", cores=threads, kind="port",
                sample=f"CPU restatement of the reference numeric phase (blocked, OpenMP) on this workload: "
                       f"the first {100 * done / tot:.1f}% of its delay-free flops ({done:.3e} of {tot:.3e}, "
                       f"bottom-up) in {t:.1f} s on {threads} threads, scaled to the whole factorization by flops "
                       f"(the full run is the reference arm, bench.py --impl reference)")


def reference_full_run(rv, orc, s, b, steps, warmup):
    """The reference arm: ONE complete factor + solve of the workload by the
    CPU restatement of the reference numeric phase, on every host core,
    timed in `steps` slices (each a bounded part of the factorization, cut by
    delay-free flops; the last one also runs the solve).  The value is the
    sum of the slices: the measured time of the whole factor + solve.  The
    warm-up steps run the first slices of a separate factorization of the
    same matrix, which is then discarded."""
    sym, sc = cpu_analyze(rv, orc, s)
    threads = cpu_threads()
    for w in range(warmup):
        f = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=threads, sliced=True)
        f.advance(f.total_flops() * 0.005 * (w + 1))
        f.close()
    orc.release_cache()
    f = orc.OracleFactor(s, sym, sc, orc.options(), nthreads=threads, sliced=True)  # pattern set-up, untimed
    tot = f.total_flops()
    times = []
    x = None
    for i in range(steps):
        t0 = time.perf_counter()
        if i < steps - 1:
            f.advance(tot * (i + 1) / steps)
        else:
            f.finish()
            x = f.solve(b)
        times.append(time.perf_counter() - t0)
    if x is None:  # steps == 0
        f.finish()
        x = f.solve(b)
    err = rv.problems.backward_error(s, x, b)
    inertia = f.inertia()
    st = f.stats()
    f.close()
    orc.release_cache()
    return dict(value=sum(times), times=times, cores=threads, bwd_err=err, inertia=inertia, stats=st, flops=tot)


class ClockSampler:
    def __init__(self):
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self, device_index=0):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or parts[0] != str(device_index):
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def gemm_peak_tflops(torch, dtype):
    """cuBLAS GEMM throughput on this GPU: FP64 (DGEMM) or TF32 (FP32 inputs, TF32 tensor math)."""
    n = 8192
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    a = torch.randn(n, n, dtype=dtype, device="cuda")
    b = torch.randn(n, n, dtype=dtype, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


def run_batch(args, rv, entry, torch, barrier, max_over_ranks, rank, world, local, dist=None):
    """The many-systems workload: 64 systems (n log-uniform in [5e3, 2e5],
    half shifted Laplacians, half KKT, seed 1) with 1-32 right-hand sides each,
    in plain FP64.  The systems form block-diagonal unions sized to the device
    memory (BatchLDLT groups); a step factors and solves every group in turn,
    releasing each group's device memory before the next.  Then
    refactorizations with every value scaled by 1 + 0.01 N(0,1) (symmetric
    pairs alike), each followed by the solve.  On N GPUs the 64 systems are
    split between the ranks (balanced by flops, no collective in the data
    path): the total work is fixed, the time is the slowest rank's."""
    t0 = time.perf_counter()
    fam = rv.problems.batch_family(count=64, seed=1)
    mine = list(range(len(fam)))
    if world > 1:
        weights = [dense_flops(rv.SparseLDLT.analyze(f[0]).symbolic) for f in fam]
        mine = rv.replicas.shard(weights, rank, world)
    systems, nrhs = [fam[i][0] for i in mine], [fam[i][1] for i in mine]
    bl = rv.BatchLDLT(systems)
    analyze_ms = (time.perf_counter() - t0) * 1e3
    flops = sum(dense_flops(g.solver.symbolic) for g in bl.groups)
    rhs = [rv.problems.rhs_normal(sy.n, 100 + i, r) for i, sy, r in zip(mine, systems, nrhs)]
    opts = rv.FactorOptions(precision="fp64")
    vals = bl.values()
    d_vals = torch.from_numpy(vals).to("cuda")
    G = []  # per group: scaling, right-hand sides (R columns of length n_g), solution buffer, stream
    scals = [torch.from_numpy(g.solver._scaling).to("cuda") for g in bl.groups]
    # each union's scheduling options tuned on its own pattern and values (plain FP64: results unchanged)
    tables = bl.autotune_groups(d_vals.data_ptr(), [t.data_ptr() for t in scals], opts, reps=1)
    for g, sc in zip(bl.groups, scals):
        big = bl.rhs_matrix(rhs, g.first, g.count)
        g.solver._ensure_handle(g.options)
        g.solver.trim(workspace=True, factor=True)  # creation sized the arenas: give them back until its turn
        g.solver.set_profiling(True)
        G.append(dict(g=g, scal=sc, R=big.shape[1],
                      rhs=torch.from_numpy(np.ascontiguousarray(big.T)).to("cuda"),
                      x=torch.empty(big.shape[1], big.shape[0], dtype=torch.float64, device="cuda"),
                      stream=torch.cuda.ExternalStream(g.solver.stream()), voff=int(bl.voffsets[g.first])))
    multi = len(bl.groups) > 1
    # symmetric perturbation map on the device: entry -> its unordered pair
    invs, base = [], 0
    for g in bl.groups:
        u = g.union
        col = np.repeat(np.arange(u.n, dtype=np.int64), np.diff(u.colptr))
        key = np.minimum(u.rowidx, col) * np.int64(u.n) + np.maximum(u.rowidx, col)
        uq, inv = np.unique(key, return_inverse=True)
        invs.append(inv.astype(np.int64) + base)
        base += uq.size
    d_inv = torch.from_numpy(np.concatenate(invs)).to("cuda")
    del invs
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    d_pert = torch.empty_like(d_vals)

    def step(dv):
        for e in G:
            g = e["g"]
            g.solver.factor_device(dv.data_ptr() + 8 * e["voff"], e["scal"].data_ptr(), g.options)
            with torch.cuda.stream(e["stream"]):  # the handle's stream orders the copy before the solve
                e["x"].copy_(e["rhs"])
            g.solver.solve_device(e["x"].data_ptr(), e["R"], g.union.n)
            if multi:
                g.solver.trim(workspace=True, factor=True)

    def timed(dv):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(G[0]["stream"]):
            e0.record(G[0]["stream"])
        step(dv)
        with torch.cuda.stream(G[-1]["stream"]):
            e1.record(G[-1]["stream"])
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    def check(values):
        errs = []
        for e in G:
            g = e["g"]
            xg = e["x"].cpu().numpy().T
            xs = bl.split(np.asfortranarray(xg), rhs, g.first, g.count)
            for i in range(g.count):
                sy = systems[g.first + i]
                lo, hi = bl.voffsets[g.first + i], bl.voffsets[g.first + i + 1]
                sv = rv.problems.System(name="v", n=sy.n, colptr=sy.colptr, rowidx=sy.rowidx, values=values[lo:hi])
                bb = rhs[g.first + i]
                bb = bb if bb.ndim == 2 else bb[:, None]
                xx = xs[i] if xs[i].ndim == 2 else xs[i][:, None]
                errs.append(max(rv.problems.backward_error(sv, xx[:, j], bb[:, j]) for j in range(bb.shape[1])))
        return max(errs)

    for _ in range(args.warmup):
        step(d_vals)
    barrier()
    clocks = ClockSampler()
    times = [timed(d_vals) for _ in range(args.steps)]
    launches = sum(e["g"].solver.profile()["factor_launches"] + e["g"].solver.profile()["solve_launches"] for e in G)
    parts = {}
    for e in G:
        for k, v in e["g"].solver.profile()["part_ms"].items():
            parts[k] = parts.get(k, 0.0) + v
    peak = max(e["g"].solver.profile()["peak_bytes"] for e in G)
    bwd = check(vals)
    nref = 20
    ref_times = []
    for r in range(nref):
        f = 1.0 + 0.01 * torch.randn(base, dtype=torch.float64, device="cuda", generator=gen)
        torch.mul(d_vals, f[d_inv], out=d_pert)
        del f
        torch.cuda.synchronize()
        ref_times.append(timed(d_pert))
    clk = clocks.stop(local)
    bwd_ref = check(d_pert.cpu().numpy())
    # the same perturbed refactorizations replayed as CUDA graphs: each union's arenas keep their addresses
    # while its memory is released between turns (graph_refactor = 2); a union whose pivoting changed is
    # refactored dynamically (the replay's device checks) and recorded anew
    for e in G:
        g = e["g"]
        g.options = dataclasses.replace(g.options, graph_refactor=2)
        g.solver._ensure_handle(g.options)  # a new handle: its own stream (the old one is destroyed)
        e["stream"] = torch.cuda.ExternalStream(g.solver.stream())
        g.solver.set_profiling(False)
        g.solver.trim(workspace=True, factor=True)
    gen.manual_seed(7)
    ngr = 4
    gr_times, replayed = [], 0
    for r in range(ngr):
        f = 1.0 + 0.01 * torch.randn(base, dtype=torch.float64, device="cuda", generator=gen)
        torch.mul(d_vals, f[d_inv], out=d_pert)
        del f
        torch.cuda.synchronize()
        gr_times.append(timed(d_pert))
        replayed += sum(1 for e in G if e["g"].solver.profile()["factor_launches"] == 1)
    bwd_gr = check(d_pert.cpu().numpy())
    for e in G:  # back to the dynamic options for the end-to-end runs
        e["g"].options = dataclasses.replace(e["g"].options, graph_refactor=0)
    # end to end through the public API with host buffers: BatchLDLT.factor_solve
    e2e_t = []
    for _ in range(max(1, min(args.steps, 2))):
        barrier()
        t1 = time.perf_counter()
        bl.factor_solve(None, rhs)  # each union with its tuned options
        torch.cuda.synchronize()
        e2e_t.append(time.perf_counter() - t1)
    inert_ok = bl.inertias() == [sy.inertia for sy in systems]
    t_step = max_over_ranks(statistics.mean(times))
    t_ref = max_over_ranks(statistics.mean(ref_times))
    e2e_v = max_over_ranks(statistics.mean(e2e_t))
    flops_all = rv.replicas.sum_over_ranks(flops, dist, device="cuda")
    n_all = int(rv.replicas.sum_over_ranks(bl.n, dist, device="cuda"))
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = entry.load_oracle()
        cb = batch_cpu_baseline(rv, orc, systems, flops)
    if rank == 0:
        ns = [sy.n for sy in systems]
        h2d = int(vals.nbytes + sum(e["rhs"].numel() * 8 for e in G))
        line = {
            "metric": "batch factor+solve time (64 systems, 1-32 RHS each), plain FP64",
            "value": t_step, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": False,
            "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded generator, no public suite)",
            "config": {"workload": CONFIGS["batch64"][2], "systems": len(fam), "systems_rank0": len(systems),
                       "n_total": n_all,
                       "n_min": min(ns), "n_max": max(ns), "rhs_total": int(sum(nrhs)),
                       "groups": [g.count for g in bl.groups],
                       "device_budget_gb": bl.device_budget / 1e9,
                       "form": "plain FP64; block-diagonal unions (one handle each) factored, solved and "
                               "released in turn",
                       "scaling": "MC64 per system (host analysis incl. ordering %.0f ms)" % analyze_ms,
                       "l2": "working set far above L2 (126 MB); no flush needed",
                       "parallelism": f"systems split over {world} GPUs" if world > 1 else "one GPU"},
            "bwd_err_max": bwd, "inertia_exact": inert_ok,
            "refactor": {"count": nref, "perturbation": "values x (1 + 0.01 N(0,1)), symmetric pairs alike",
                         "s_per_refactor_mean": t_ref, "s_min": min(ref_times),
                         "s_max": max(ref_times), "bwd_err_max_last": bwd_ref},
            "refactor_graph": {"count": ngr, "perturbation": "the first %d of the same sequence" % ngr,
                               "s_per_refactor_mean": max_over_ranks(statistics.mean(gr_times)),
                               "s_per_refactor_after_capture": max_over_ranks(statistics.mean(gr_times[2:])),
                               "union_factorizations_replayed": replayed,
                               "union_factorizations": ngr * len(G), "bwd_err_max_last": bwd_gr,
                               "how": "graph_refactor = 2 (arenas at fixed addresses across rvg_trim); the first "
                                      "refactorization records, the second captures, later ones replay while the "
                                      "pivoting stays the same (with 1% random perturbations it changes in some "
                                      "system of every union, and the device checks fall back to the dynamic path)"},
            "factor_flops": flops_all, "factor_gflops": flops_all / t_step / 1e9,
            "e2e": {"value": e2e_v, "unit": "s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(sum(e["rhs"].numel() * 8 for e in G))},
            "gpu_launches": int(launches),
            "autotune": [{"group": gi, "chosen": {"large_front_threshold": g.options.large_front_threshold,
                                                  "mixed_tile_cols": g.options.mixed_tile_cols},
                          "candidates": [dict(c, factor_s=t) for c, t in tab]}
                         for gi, (g, tab) in enumerate(zip(bl.groups, tables))],
            "parts_ms": parts, "step_event_s": times, "peak_device_bytes": peak, "clocks": clk,
            "cpu_baseline": cb,
        }
        print(json.dumps(line), flush=True)
    bl.close()


def batch_cpu_baseline(rv, orc, systems, full_flops, budget_s=10.0):
    """The CPU restatement on the first systems of the batch (a bounded
    sample, all host cores), scaled to the whole batch by flops."""
    threads = cpu_threads()
    t, fl, used = 0.0, 0.0, 0
    for sy in systems:
        if t > budget_s:
            break
        sym, sc = cpu_analyze(rv, orc, sy)
        b = rv.problems.rhs_normal(sy.n, 0)
        t0 = time.perf_counter()
        f = orc.OracleFactor(sy, sym, sc, orc.options(), nthreads=threads)
        f.solve(b)
        t += time.perf_counter() - t0
        f.close()
        fl += dense_flops(sym)
        used += 1
    orc.release_cache()
    rate = fl / t
    return dict(value=full_flops / rate, unit="s", cores=threads, kind="port",
                sample=f"CPU restatement, factor+solve of the first {used} systems: {t:.2f} s for {fl:.3e} flops "
                       f"({rate / 1e9:.1f} GFLOP/s), scaled to the batch's {full_flops:.3e} flops")


def time_form(rv, torch, solver, s, b, opts, warmup, steps):
    """Factor + solve to 1e-14 (refinement escalating to GMRES-IR) with the
    values, scaling and right-hand side resident on the device; CUDA events on
    the handle's stream around each step.  Returns the mean step time and the
    last step's accuracy figures."""
    solver._ensure_handle(opts)
    st = torch.cuda.ExternalStream(solver.stream())
    d_vals = torch.from_numpy(s.values).to("cuda")
    d_scal = torch.from_numpy(solver._scaling).to("cuda") if solver._scaling is not None else None
    d_b = torch.from_numpy(b).to("cuda")
    d_x = torch.empty_like(d_b)
    out = {}

    def step():
        solver.factor_device(d_vals.data_ptr(), d_scal.data_ptr() if d_scal is not None else None, opts)
        return solver.solve_auto_device(d_b.data_ptr(), d_x.data_ptr(), tol=1e-14, max_iter=100)

    for _ in range(warmup):
        step()
    times, its, used = [], [], set()
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        it, err, how = step()
        e1.record(st)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
        its.append(it)
        used.add(how)
    out.update(s_per_step=statistics.mean(times), times=times, solves_after_first=its, methods=sorted(used),
               bwd_err=rv.problems.backward_error(s, d_x.cpu().numpy(), b), inertia=list(solver.inertia()))
    if opts.precision == "learned":
        out["selector"] = solver.selector_stats()
    return out


def run_learned(args, rv, torch):
    """The selector workload: label the generated training family on the GPU
    (every matrix factored with all large fronts in FP64 and all in the mixed
    form), train the network with the library's kernels, then time plain
    FP64, the mixed form and the learned form on held-out matrices."""
    S = rv.selector
    t0 = time.perf_counter()
    fam = S.c5_family(args.train_count, 11, 20, 60)
    lab_opts = rv.FactorOptions(large_front_threshold=256, mixed_flush=0, mixed_operands="bf16")
    data = S.label_family(fam, 1e-3, lab_opts)
    t_label = time.perf_counter() - t0
    sel = S.PrecisionSelector(seed=11)
    sel.fit_normalisation(data.X)
    t1 = time.perf_counter()
    hist = sel.train(data.X, data.y, weights=S.sample_weights(data, 0.5), steps=3000, lr=3e-3)
    t_train = time.perf_counter() - t1
    held = [rv.problems.shifted_laplacian(100, 0.05),
            rv.problems.kkt(60, seed=20261203, reg_hi=10.0 ** -5)]
    rows, clocks = [], ClockSampler()
    for s in held:
        solver, an_ms = analyze(rv, s)
        solver.set_selector(sel)
        b = rv.problems.rhs_normal(s.n, seed=1)
        r = {"matrix": s.name, "n": s.n, "analyze_ms": an_ms}
        for form in ("fp64", "mixed", "learned"):
            o = rv.FactorOptions(precision=form, mixed_flush=0, mixed_operands="bf16")
            r[form] = time_form(rv, torch, solver, s, b, o, args.warmup, args.steps)
        solver.close()
        X, y, err, m = S.label_fronts(s, 1e-3, rv.FactorOptions(mixed_flush=0, mixed_operands="bf16"))
        r["misprediction"] = S.misprediction(sel, S.Labelled(X, y, err, m, [0] * y.size))
        rows.append(r)
        torch.cuda.empty_cache()
    clk = clocks.stop(0)
    for r in rows:  # the 2x target (learned at least twice as fast as plain FP64) per matrix
        sp = r["fp64"]["s_per_step"] / r["learned"]["s_per_step"]
        r["learned_vs_plain_fp64"] = sp
        r["learned_vs_all_mixed"] = r["mixed"]["s_per_step"] / r["learned"]["s_per_step"]
        sel_st = r["learned"].get("selector", {})
        r["target_2x"] = "met" if sp >= 2.0 else (
            "not met: all-mixed is %.2fx plain FP64 here (%d solves after the first against %d for plain FP64); "
            "the selector sent %s of %s large fronts to the mixed form" % (
                r["fp64"]["s_per_step"] / r["mixed"]["s_per_step"], max(r["mixed"]["solves_after_first"]),
                max(r["fp64"]["solves_after_first"]), sel_st.get("routed_mixed"), sel_st.get("large_fronts")))
    t_l = sum(r["learned"]["s_per_step"] for r in rows)
    t_p = sum(r["fp64"]["s_per_step"] for r in rows)
    t_m = sum(r["mixed"]["s_per_step"] for r in rows)
    line = {"metric": METRIC, "value": t_l, "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_l * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": form_dtype(rv.FactorOptions(precision="learned", mixed_flush=0, mixed_operands="bf16")),
            "data": "synthetic (seeded generators; held-out seeds for evaluation)",
            "config": {"workload": CONFIGS["learned"][2], "form": "learned: BF16-part tensor-core Schur updates on "
                       "the fronts the selector predicts safe, plain FP64 elsewhere; refinement escalating to "
                       "GMRES-IR", "value": "sum over the held-out matrices of factor+solve time to 1e-14",
                       "l2": "working sets far above L2 (126 MB); no flush needed"},
            "sum_fp64_s": t_p, "sum_mixed_s": t_m, "speedup_vs_plain_fp64": t_p / t_l,
            "speedup_vs_all_mixed": t_m / t_l, "held_out": rows,
            "kkt80": "not run: the KKT on an 80^3 H does not fit one B200 (see the default line's configs); "
                     "the 60^3 KKT stands in for it",
            "training": {"matrices": len(fam), "fronts": int(data.y.size), "safe_fraction": float(data.y.mean()),
                         "tau": 1e-3, "label_s": t_label, "train_s": t_train, "adam_steps": 3000,
                         "loss_first": hist[0][1], "loss_last": hist[-1][1],
                         "train_misprediction": S.misprediction(sel, data)},
            "clocks": clk}
    print(json.dumps(line), flush=True)


def choose_form(forms: dict, plain: str = "plain_fp64", tol: float = 1e-14):
    """The fastest form whose backward error reaches tol and whose inertia
    equals the plain FP64 form's (exact); the plain form always qualifies.
    forms: name -> {"t": seconds, "bwd": backward error, "inertia": (p, n, z)}."""
    ref = list(forms[plain]["inertia"])
    ok = [k for k, f in forms.items() if k == plain or (f["bwd"] <= tol and list(f["inertia"]) == ref)]
    return min(ok, key=lambda k: forms[k]["t"])


def form_dtype(opts):
    """The arithmetic a form computes in (not a precision claim: every form
    reaches the same 1e-14 backward error)."""
    if opts.precision == "fp64":
        return "f64"
    parts = "bf16x3" if opts.mixed_operands == "bf16" else "tf32x3"
    lead = "learned per front: f64 or " if opts.precision == "learned" else ""
    return f"{lead}{parts} Schur products, fp32 accumulation (fp64 sums), fp64 pivoting/storage/solve, fp64 refinement"


def side_config(rv, torch, name, s, b, warmup, steps, selector=None, bf16_opts=None):
    """A further configuration on the same line: plain FP64, the BF16 mixed
    form and the learned form, each factor + solve to 1e-14 with inputs in
    HBM (W warm-up, K timed steps); the fastest accurate one is its value.
    One extra profiled step of that form gives its Schur-GEMM rate."""
    t0 = time.perf_counter()
    solver, an_ms = analyze(rv, s)
    if selector is not None:
        solver.set_selector(selector)
    forms = {"plain_fp64": rv.FactorOptions(precision="fp64"),
             "mixed_bf16_flush0": bf16_opts or rv.FactorOptions(precision="mixed", mixed_flush=0,
                                                                  mixed_operands="bf16")}
    if selector is not None:
        forms["learned_bf16_flush0"] = rv.FactorOptions(precision="learned", mixed_flush=0, mixed_operands="bf16")
    res = {}
    for k, o in forms.items():
        r = time_form(rv, torch, solver, s, b, o, warmup, steps)
        res[k] = {"s_per_step": r["s_per_step"], "bwd_err": r["bwd_err"], "inertia": r["inertia"],
                  "solves_after_first": r["solves_after_first"], "methods": r["methods"]}
        if "selector" in r:
            res[k]["selector"] = r["selector"]
    # the fastest accurate form with the plain form's (exact) inertia
    chosen = choose_form({k: {"t": r["s_per_step"], "bwd": r["bwd_err"], "inertia": r["inertia"]}
                          for k, r in res.items()})
    solver._ensure_handle(forms[chosen])
    solver.set_profiling(True)
    time_form(rv, torch, solver, s, b, forms[chosen], 0, 1)
    pr = solver.profile()
    solver.set_profiling(False)
    work = solver.work()
    solver.close()
    torch.cuda.empty_cache()
    c = res[chosen]
    gemm = None
    if pr["syrk_ms"] > 0:
        gemm = {"tflops_fp64_equiv": pr["syrk_flops"] / (pr["syrk_ms"] * 1e-3) / 1e12,
                "share_of_step": pr["syrk_ms"] * 1e-3 / c["s_per_step"], "launches": pr["syrk_launches"]}
    return {"workload": name, "n": s.n, "value": c["s_per_step"], "unit": "s", "chosen_form": chosen,
            "dtype": form_dtype(forms[chosen]), "bwd_err": c["bwd_err"], "inertia": c["inertia"],
            "inertia_expected": list(s.inertia), "inertia_exact": list(c["inertia"]) == list(s.inertia),
            "speedup_vs_plain_fp64": res["plain_fp64"]["s_per_step"] / c["s_per_step"],
            "forms": res, "schur_gemm": gemm, "factor_gflops": work["flops_factor"] / c["s_per_step"] / 1e9,
            "solve_gbs_per_rhs": None, "analyze_ms": an_ms, "wall_s": time.perf_counter() - t0,
            "steps": steps, "warmup": warmup}


def batch_subset(rv, torch, count, warmup, steps):
    """The first `count` systems of the many-systems workload (64 systems, n
    log-uniform in [5e3, 2e5] from seed 1, 1-32 RHS each), plain FP64, end
    to end through BatchLDLT.factor_solve (values and right-hand sides from
    host memory, solutions back): a bounded part of that workload."""
    fam = rv.problems.batch_family(count=64, seed=1)[:count]
    systems, nrhs = [f[0] for f in fam], [f[1] for f in fam]
    rhs = [rv.problems.rhs_normal(sy.n, 100 + i, r) for i, (sy, r) in enumerate(zip(systems, nrhs))]
    bl = rv.BatchLDLT(systems)
    opts = rv.FactorOptions(precision="fp64")
    for _ in range(warmup):
        bl.factor_solve(None, rhs, opts)
    times = []
    for _ in range(steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xs = bl.factor_solve(None, rhs, opts)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    errs = []
    for sy, bb, xx in zip(systems, rhs, xs):
        bb2 = bb if bb.ndim == 2 else bb[:, None]
        xx2 = xx if xx.ndim == 2 else xx[:, None]
        errs.append(max(rv.problems.backward_error(sy, xx2[:, j], bb2[:, j]) for j in range(bb2.shape[1])))
    inert_ok = bl.inertias() == [sy.inertia for sy in systems]
    flops = sum(dense_flops(g.solver.symbolic) for g in bl.groups)
    bl.close()
    torch.cuda.empty_cache()
    return {"workload": f"first {count} of the 64-system batch (n {min(sy.n for sy in systems)}-"
                        f"{max(sy.n for sy in systems)}, {sum(nrhs)} right-hand sides), plain FP64, end to end",
            "value": statistics.mean(times), "unit": "s", "bwd_err_max": max(errs), "inertia_exact": inert_ok,
            "factor_gflops": flops / statistics.mean(times) / 1e9, "steps": steps, "warmup": warmup}


def run_profile_step(args, rv, torch):
    """One form on one system, W warm-up and K timed steps (factor + solve to
    1e-14 with inputs in HBM), then one step with the library's per-launch
    events: the command the committed ncu summaries were taken with."""
    s, b = build_system(rv, args.config)
    solver, _ = analyze(rv, s)
    form = {"plain": dict(precision="fp64"),
            "tf32": dict(precision="mixed", mixed_flush=4, mixed_operands="tf32"),
            "bf16": dict(precision="mixed", mixed_flush=0, mixed_operands="bf16"),
            "learned": dict(precision="learned", mixed_flush=0, mixed_operands="bf16")}[args.profile_step]
    if args.profile_step == "learned":
        solver.set_selector(rv.PrecisionSelector.load(SELECTOR))
    opts = rv.FactorOptions(far_field_sms=args.far_sms, mixed_window=args.mixed_window, **form)
    r = time_form(rv, torch, solver, s, b, opts, args.warmup, args.steps)
    p0 = solver.profile()  # host counters of the last timed step (no per-launch events)
    host = {k: p0[k] for k in ("host_total_ms", "host_sync_ms", "host_wait_ms", "host_gap_ms", "lf_misses")}
    solver.set_profiling(True)
    time_form(rv, torch, solver, s, b, opts, 0, 1)
    pr = solver.profile()
    solver.close()
    print(json.dumps({"config": args.config, "form": args.profile_step, "n": s.n, "s_per_step": r["s_per_step"],
                      "bwd_err": r["bwd_err"], "inertia": r["inertia"], "solves_after_first": r["solves_after_first"],
                      "phases_ms": {k: pr[k] for k in ("factor_ms", "solve_ms", "assembly_ms", "host_sync_ms",
                                                       "host_wait_ms")},
                      "timed_step_host": host,
                      "schur_gemm": {"ms": pr["syrk_ms"], "flops_fp64_equiv": pr["syrk_flops"],
                                     "launches": pr["syrk_launches"]},
                      "parts_ms": pr["part_ms"]}), flush=True)


def run_reference(args, rv, entry, rank):
    """The reference arm: the CPU restatement of the reference's numeric phase
    (oracle/, OpenMP, all host cores) on this arm's workload, through the
    oracle's own libraries only (its analysis library reuses the library's
    host analysis sources without the GPU code).  Rank 0 alone runs it."""
    if rank != 0:
        return
    orc = entry.load_oracle()
    threads = cpu_threads()
    base = {"metric": METRIC, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "impl": "reference"}
    if args.config in ("batch64", "learned"):
        # bounded samples of these workloads, scaled by flops
        if args.config == "batch64":
            systems = [f[0] for f in rv.problems.batch_family(count=64, seed=1)]
            full = sum(dense_flops(cpu_analyze(rv, orc, sy)[0]) for sy in systems)
            cb = batch_cpu_baseline(rv, orc, systems, full)
        else:
            parts = []
            for cfg in ("lap100", "kkt60"):
                s, b = build_system(rv, cfg)
                parts.append(cpu_sample(rv, orc, s, b))
            cb = dict(parts[1])
            cb["value"] = parts[0]["value"] + parts[1]["value"]
            cb["sample"] = "; ".join(p["sample"] for p in parts) + " (sum of the two)"
        v = cb["value"]
        line = dict(base, value=v, ms_per_step=v * 1e3,
                    config={"workload": CONFIGS[args.config][2], "form": "plain FP64 (CPU restatement)",
                            "timing": "bounded sample scaled by flops"},
                    cpu_baseline=cb, e2e={"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return
    s, b = build_system(rv, args.config)
    r = reference_full_run(rv, orc, s, b, max(args.steps, 1), args.warmup)
    v = r["value"]
    sample = (f"one complete factor+solve of this workload ({r['flops']:.3e} delay-free flops after amalgamation), "
              f"timed in {len(r['times'])} slices cut by flops (the last with the solve); value = their sum")
    line = dict(base, value=v, ms_per_step=1e3 * v / len(r["times"]),
                config={"workload": CONFIGS[args.config][2],
                        "form": "plain FP64, CPU restatement of the reference numeric phase (blocked rank-32 "
                                "updates, OpenMP inside large fronts and across each wave's fronts)",
                        "ordering": "geometric nested dissection, constraints last", "scaling": "MC64",
                        "timing": "steps are consecutive slices of ONE factorization; value = sum of the slices",
                        "l2": "working set far above the CPU caches"},
                step_s=r["times"], bwd_err=r["bwd_err"], inertia=list(r["inertia"]), stats=r["stats"],
                factor_gflops=r["flops"] / v / 1e9,
                cpu_baseline={"value": v, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
                e2e={"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="kkt60", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-precision form")
    ap.add_argument("--no-side", action="store_true",
                    help="default workload only: skip the C1, C4 Laplacian and C3-subset measurements")
    ap.add_argument("--train-count", type=int, default=200, help="learned config: generated training matrices")
    ap.add_argument("--mixed-flush", default="4,0",
                    help="comma list of mixed-form flush depths to time (32-deep K chunks per FP32 partial sum; 0 = all K)")
    ap.add_argument("--profile-step", default=None, choices=["plain", "tf32", "bf16", "learned"],
                    help="profiling aid: time only this form (factor + solve to 1e-14) on --config and print "
                         "its time and parts; no contract line")
    ap.add_argument("--mixed-window", type=int, default=0,
                    help="--profile-step: outer blocks per window of deferred mixed-form updates (0 = default)")
    ap.add_argument("--far-sms", type=int, default=-1,
                    help="profiling step: SMs a window's far-field update leaves to the next blocks (0 = no split)")
    ap.add_argument("--bf16-flush", default="0",
                    help="the same for the mixed form with BF16 operand parts")
    args = ap.parse_args()
    if not args.profile_step:
        args.warmup = max(args.warmup, 3)

    import __graft_entry__ as entry
    rv = entry.load_package()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rv, entry, rank)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.profile_step:
        run_profile_step(args, rv, torch)
        return
    if args.config == "learned":
        if rank == 0:
            run_learned(args, rv, torch)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.config == "batch64":
        run_batch(args, rv, entry, torch, barrier, max_over_ranks, rank, world, local, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    s, b = build_system(rv, args.config)
    solver, analyze_ms = analyze(rv, s)
    full_flops = dense_flops(solver.symbolic)
    d_scal = torch.from_numpy(solver._scaling).to("cuda") if solver._scaling is not None else None
    d_vals = torch.from_numpy(s.values).to("cuda")
    d_b = torch.from_numpy(b).to("cuda")
    d_x = torch.empty_like(d_b)

    def run_form(precision, flush=4, ops="tf32", method="ir", **extra):
        """W warm-up + K timed steps of one form: factor + (refined) solve, inputs in HBM.
        method: "ir" (iterative refinement) or "gmres" (GMRES-IR) back to FP64 accuracy."""
        opts = rv.FactorOptions(precision=precision, mixed_flush=flush, mixed_operands=ops, **extra)
        used = set()
        solver._ensure_handle(opts)
        solver.set_profiling(False)  # timed steps without the per-launch events
        stream = torch.cuda.ExternalStream(solver.stream())

        def step():
            solver.factor_device(d_vals.data_ptr(), d_scal.data_ptr() if d_scal is not None else None, opts)
            if method == "gmres":
                return solver.solve_gmres_device(d_b.data_ptr(), d_x.data_ptr(), tol=1e-14, max_iter=100, restart=30)
            if method == "auto":
                it, e, how = solver.solve_auto_device(d_b.data_ptr(), d_x.data_ptr(), tol=1e-14, max_iter=100)
                used.add(how)
                return it, e
            return solver.solve_refine_device(d_b.data_ptr(), d_x.data_ptr(), tol=1e-14, max_iter=10)

        for _ in range(args.warmup):
            step()
        barrier()
        clocks = ClockSampler()
        times, walls, launches, its = [], [], 0, []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
            w0 = time.perf_counter()
            it, _ = step()
            walls.append(time.perf_counter() - w0)
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
            pr = solver.profile()
            launches += pr["factor_launches"] + pr["solve_launches"] * (1 + it)
            its.append(it)
        barrier()
        clk = clocks.stop(local)
        # one more step with the per-launch events on: where the time goes, the Schur GEMM's rate
        solver.set_profiling(True)
        step()
        pr = solver.profile()
        solver.set_profiling(False)
        syrk_ms, syrk_flops, syrk_launch = pr["syrk_ms"], pr["syrk_flops"], pr["syrk_launches"]
        x = d_x.cpu().numpy()
        return dict(t=max_over_ranks(statistics.mean(times)), times=times, walls=walls, clk=clk,
                    bwd=rv.problems.backward_error(s, x, b), inertia=solver.inertia(), stats=solver.stats(),
                    prof=solver.profile(), syrk_ms=syrk_ms, syrk_flops=syrk_flops, syrk_launch=syrk_launch,
                    launches=launches, refine_iters=its, opts=opts, method=method, used=sorted(used))

    plain = run_form("fp64")
    forms = {"plain_fp64": plain}
    for fl in [int(v) for v in args.mixed_flush.split(",") if v.strip()]:
        forms[f"mixed_flush{fl}"] = run_form("mixed", fl, "tf32", "auto")
    # the scheduling options of the BF16 form tuned on this pattern (results do not depend on them)
    # and its window depth, which changes the arithmetic: a deeper window only with a faster factor + solve
    # and the plain form's inertia
    def window_step(o):
        r = time_form(rv, torch, solver, s, b, o, 1, 1)
        return r["s_per_step"], r["inertia"]
    tuned, tune_table = rv.autotune.autotune(solver, d_vals.data_ptr(), d_scal.data_ptr() if d_scal is not None else None,
                                             rv.FactorOptions(precision="mixed", mixed_flush=0, mixed_operands="bf16"),
                                             reps=1, step=window_step, expect_inertia=plain["inertia"])
    autotune_rep = {"candidates": [dict(c, **({"step_s": s_} if c.get("step") else {"factor_s": s_}))
                                   for c, s_ in tune_table],
                    "chosen": {"large_front_threshold": tuned.large_front_threshold,
                               "mixed_tile_cols": tuned.mixed_tile_cols, "mixed_window": tuned.mixed_window}}
    for fl in [int(v) for v in args.bf16_flush.split(",") if v.strip()]:
        extra = ({"large_front_threshold": tuned.large_front_threshold, "mixed_tile_cols": tuned.mixed_tile_cols,
                  "mixed_window": tuned.mixed_window} if fl == 0 else {})
        forms[f"mixed_bf16_flush{fl}"] = run_form("mixed", fl, "bf16", "auto", **extra)
    if os.path.exists(SELECTOR) and not args.no_learned:
        # the shipped selector picks the form per large front (BF16 parts where it predicts safe, FP64 elsewhere)
        solver.set_selector(rv.PrecisionSelector.load(SELECTOR))
        forms["learned_bf16_flush0"] = run_form("learned", 0, "bf16", "auto")
        forms["learned_bf16_flush0"]["selector"] = solver.selector_stats()
    # the chosen form: the fastest that reaches the accuracy target with the plain form's inertia
    chosen_key = choose_form(forms)
    chosen = forms[chosen_key]
    chosen_name = "plain" if chosen_key == "plain_fp64" else "mixed"
    t_step = chosen["t"]
    syrk_ms, syrk_flops, syrk_launch, launches = (plain["syrk_ms"], plain["syrk_flops"], plain["syrk_launch"],
                                                   chosen["launches"])
    clk = chosen["clk"]
    bwd, inertia, stats, prof = chosen["bwd"], chosen["inertia"], chosen["stats"], chosen["prof"]
    times, walls = chosen["times"], chosen["walls"]

    # end to end through the public API with host buffers (the chosen form): values and right-hand side in
    # pinned host memory, copied to the device inside the timed region by rvg_factor / the solve, the solution
    # copied back; one untimed call first (the handle for these options and its arenas are set up there)
    e2e_times = []
    xh = None
    opts = chosen["opts"]
    solver._ensure_handle(opts)
    vals_pinned = torch.from_numpy(s.values).pin_memory().numpy()
    b_pinned = torch.from_numpy(b).pin_memory().numpy()
    for it in range(1 + max(1, min(args.steps, 3))):
        barrier()
        t0 = time.perf_counter()
        solver.factor(vals_pinned, opts)
        if chosen["method"] == "gmres":
            xh, _, _ = solver.solve_gmres(b_pinned, tol=1e-14, max_iter=100, restart=30)
        elif chosen["method"] == "auto":
            xh, _, _, _ = solver.solve_auto(b_pinned, tol=1e-14, max_iter=100)
        else:
            xh, _, _ = solver.solve_refine(b_pinned, tol=1e-14, max_iter=10)
        torch.cuda.synchronize()
        if it > 0:
            e2e_times.append(time.perf_counter() - t0)
    e2e = max_over_ranks(statistics.mean(e2e_times))
    bwd_e2e = rv.problems.backward_error(s, xh, b)

    # blocked multi-RHS solve: 8 right-hand sides in one call against 8 single calls (device-resident)
    stream = torch.cuda.ExternalStream(solver.stream())
    rhs8 = torch.randn(8, s.n, dtype=torch.float64, device="cuda")  # 8 columns of length n, ld n
    def timed(fn):
        for _ in range(2):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)
    multi = {"nrhs": 8,
             "blocked_ms": timed(lambda: solver.solve_device(rhs8.data_ptr(), 8, s.n)),
             "one_at_a_time_ms": timed(lambda: [solver.solve_device(rhs8[r].data_ptr(), 1, s.n) for r in range(8)])}

    # refactorization (factor only, same pattern and values): dynamic against replayed as one CUDA graph
    def factor_times(o, reps):
        solver._ensure_handle(o)  # other options: a new handle, with a stream of its own
        fst = torch.cuda.ExternalStream(solver.stream())
        out, launches = [], []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(fst)
            solver.factor_device(d_vals.data_ptr(), d_scal.data_ptr() if d_scal is not None else None, o)
            e1.record(fst)
            e1.synchronize()
            out.append(e0.elapsed_time(e1) * 1e-3)
            launches.append(solver.profile()["factor_launches"])
        return out, launches
    o_dyn = chosen["opts"]
    t_dyn, l_dyn = factor_times(o_dyn, 3)
    t_rep, l_rep = factor_times(dataclasses.replace(o_dyn, graph_refactor=True), 5)  # records, captures, replays
    graph_refactor = {"form": chosen_key, "dynamic_factor_s": statistics.mean(t_dyn),
                      "dynamic_launches": l_dyn[-1], "replay_factor_s": statistics.mean(t_rep[2:]),
                      "first_capture_s": t_rep[1], "replayed": all(x == 1 for x in l_rep[2:])}
    solver._ensure_handle(o_dyn)
    work = solver.work()
    # the HBM-bound parts against the measured copy bandwidth: one solve (multi_rhs_solve's single-RHS
    # calls; the solve reads the factor once per RHS) and the assembly of the chosen form's profiled step
    hbm = None
    mp = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        hbm = json.load(open(mp)).get("hbm_gbs")
    t_solve1 = multi["one_at_a_time_ms"] / 8 * 1e-3
    solve_gbs = work["bytes_solve_per_rhs"] / t_solve1 / 1e9
    asm_gbs = work["bytes_assembly"] / (prof["assembly_ms"] * 1e-3) / 1e9 if prof["assembly_ms"] > 0 else None
    hbm_parts = {"peak_gbs": hbm, "peak_source": "measured-peaks file (copy)" if hbm else None,
                 "solve": {"bytes_per_rhs": work["bytes_solve_per_rhs"], "ms_per_rhs": t_solve1 * 1e3,
                           "gbs": solve_gbs, "frac": solve_gbs / hbm if hbm else None},
                 "assembly": {"bytes": work["bytes_assembly"], "ms": prof["assembly_ms"], "gbs": asm_gbs,
                              "frac": asm_gbs / hbm if (hbm and asm_gbs) else None}}
    dpeak = gemm_peak_tflops(torch, torch.float64)
    tpeak = gemm_peak_tflops(torch, torch.float32)
    # The dominant kernel's rate on ALGORITHMIC flops: the Schur-GEMM launches' FP64-equivalent work (2 K per
    # lower output entry; the mixed form executes 3 products per term, reported beside as "executed")
    syrk_ms, syrk_flops, syrk_launch = chosen["syrk_ms"], chosen["syrk_flops"], chosen["syrk_launch"]
    products = 1.0
    if chosen_name == "mixed":
        products = 3.0
        peak = tpeak
        if chosen["opts"].mixed_operands == "bf16":
            mp = os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")
            if os.path.exists(mp):
                peak = json.load(open(mp))["bf16_tflops_sustained"]
                rl_source = "measured-peaks file: cuBLAS bf16 GEMM, sustained (the kernel runs inside a long step)"
            else:
                peak = gemm_peak_tflops(torch, torch.bfloat16)
                rl_source = "cuBLAS BF16 GEMM 8192^3 measured in this run"
            rl_kernel = ("k_syrk_tc%s (mixed-form Schur GEMM: tcgen05 kind::f16, operands split into BF16 hi+lo, "
                         "3 products per term)" % ("_pair" if chosen["opts"].mixed_flush == 0 else ""))
        else:
            rl_kernel = ("k_syrk_tc%s (mixed-form Schur GEMM: tcgen05 kind::tf32, operands split hi+lo, 3 products "
                         "per term)" % ("_pair" if chosen["opts"].mixed_flush == 0 else ""))
            rl_source = "cuBLAS TF32 GEMM 8192^3 (FP32 inputs, TF32 tensor math) measured in this run"
    else:
        peak = dpeak
        rl_kernel = "k_syrk_dmma (FP64 Schur-complement GEMM, plain form)"
        rl_source = "cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in the measured-peaks file)"
    achieved = (syrk_flops / (syrk_ms * 1e-3) / 1e12) if syrk_ms > 0 else None
    # DRAM traffic per launch: ncu dram__bytes_read.sum + dram__bytes_write.sum summed over EVERY k_syrk_tc_pair
    # launch of one factorization of this workload (the BF16 form, one pass, full size), per window depth:
    # (bytes, FP64-equivalent flops) of that factorization, applied to this run's average launch
    captured = {4: (970.0e9, 8.62055e13, 712), 8: (818.1e9, 8.59948e13, 591)}
    traffic = traffic_src = None
    win = (chosen["opts"].mixed_window or 4) if chosen_name == "mixed" else None
    if chosen_name == "mixed" and chosen["opts"].mixed_operands == "bf16" and chosen["opts"].mixed_flush == 0 \
            and chosen["syrk_launch"] and args.config == "kkt60" and win in captured:
        gb, fl, nl = captured[win]
        traffic = gb / fl * (chosen["syrk_flops"] / chosen["syrk_launch"])
        traffic_src = ("ncu dram__bytes_read.sum + dram__bytes_write.sum over every k_syrk_tc_pair<BF16> launch of "
                       "one factorization of this workload at window depth %d (%.1f GB over %d launches for %.4g "
                       "FP64-equivalent flops), at this run's average launch" % (win, gb / 1e9, nl, fl))
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = entry.load_oracle()
        cb = cpu_sample(rv, orc, s, b)

    if rank == 0:
        line = {
            "metric": METRIC, "value": t_step, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": form_dtype(chosen["opts"]),
            "data": "synthetic (seeded generator, no public suite)",
            "config": {"workload": CONFIGS[args.config][2],
                       "form": (f"{chosen_key}: " + (("Schur updates on tcgen05 tensor cores (FP64 operands split "
                                "into %s hi+lo, FP32 accumulation added in FP64), FP64 pivoting/storage; FP64 "
                                "iterative refinement escalating to GMRES-IR (used: %s)"
                                % (chosen["opts"].mixed_operands.upper(), ", ".join(chosen["used"])))
                                if chosen_name == "mixed" else "plain FP64 (DMMA)")
                                + "; APTP u=0.01, nb=256, ib=32, nemin=32"),
                       "ordering": "geometric nested dissection, constraints last", "rhs": 1,
                       "scaling": "MC64 (host analysis incl. ordering %.0f ms, outside the timed region)" % analyze_ms,
                       "l2": "working set far above L2 (126 MB); no flush needed",
                       "parallelism": f"replicas x{world}"},
            "bwd_err": bwd, "bwd_err_e2e": bwd_e2e, "inertia": list(inertia), "inertia_expected": list(s.inertia),
            "forms": {k: {"s_per_step": f["t"], "bwd_err": f["bwd"], "refine_corrections": f["refine_iters"],
                          "accuracy_method": {"gmres": "GMRES-IR (FP64 FGMRES, factor as preconditioner)",
                                              "auto": "iterative refinement, escalating to GMRES-IR when it stalls "
                                                      "(used: %s)" % ", ".join(f["used"]),
                                              "ir": "iterative refinement"}[f["method"]],
                          "solves_after_first": f["refine_iters"],
                          "inertia": list(f["inertia"]),
                          "syrk_tflops_fp64_equiv": (f["syrk_flops"] / (f["syrk_ms"] * 1e-3) / 1e12)
                          if f["syrk_ms"] > 0 else None,
                          "syrk_share": (f["syrk_ms"] * 1e-3) / f["t"] if f["t"] else None,
                          "selector": f.get("selector")}
                      for k, f in forms.items()},
            "chosen_form": chosen_key,
            "speedup_vs_plain_fp64": plain["t"] / t_step,
            "stats": stats, "factor_flops": full_flops,
            "factor_gflops": full_flops / t_step / 1e9,
            "multi_rhs_solve": multi,
            "hbm_bound_parts": hbm_parts,
            "graph_refactor": graph_refactor,
            "autotune": autotune_rep,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": int(s.values.nbytes + b.nbytes),
                    "d2h_bytes_per_step": int(b.nbytes)},
            "gpu_launches": int(launches // max(args.steps, 1)),
            "roofline": {"kernel": rl_kernel, "bound": "tensor",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "achieved_unit_note": "FP64-equivalent algorithmic flops (2 K per lower output entry)",
                         "executed": {"tflops": achieved * products if achieved else None,
                                      "frac": (achieved * products / peak) if achieved else None,
                                      "products_per_term": products},
                         "traffic_unit": "bytes per launch", "traffic_source": traffic_src,
                         "peak_source": rl_source, "dgemm_peak": dpeak, "tf32_gemm_peak": tpeak,
                         "launches_per_step": syrk_launch,
                         "share_of_step": (syrk_ms * 1e-3) / t_step if t_step else None},
            "phases_ms": {k: prof[k] for k in ("factor_ms", "solve_ms", "assembly_ms", "dense_ms", "cbgemm_ms",
                                               "host_total_ms", "host_alloc_ms", "host_sync_ms", "host_wait_ms",
                                               "host_gap_ms")},
            "phases_note": ("host_sync_ms: the host blocked at each wave boundary while the device runs the wave "
                            "(it needs the wave's eliminated counts to lay out the next one); host_wait_ms: the "
                            "large-front threads blocked behind outer blocks issued ahead (summed over threads); "
                            "host_gap_ms: the only time the device has nothing of the factorization queued"),
            "lf_blocks_reissued": prof["lf_misses"],
            "parts_ms": prof["part_ms"],
            "work": work,
            "step_wall_s": walls, "step_event_s": times,
            "peak_device_bytes": prof["peak_bytes"],
            "clocks": clk,
            "cpu_baseline": cb,
        }
    solver.close()
    del d_vals, d_b, d_x, d_scal
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and args.config == "kkt60" and not args.no_side:
        # the other configurations, each with its own measured value, accuracy and inertia
        sel = rv.PrecisionSelector.load(SELECTOR) if os.path.exists(SELECTOR) else None
        k = max(1, min(args.steps, 3))
        side = {}
        s1, b1 = build_system(rv, "lap16")
        side["C1_laplace16"] = side_config(rv, torch, CONFIGS["lap16"][2], s1, b1, 3, k, sel)
        s4, b4 = build_system(rv, "lap100")
        side["C4_laplace100"] = side_config(rv, torch, CONFIGS["lap100"][2], s4, b4, 3, k, sel)
        del s4, b4
        side["C3_first8"] = batch_subset(rv, torch, 8, 1, k)
        side["C4_kkt80"] = {"unavailable": "KKT on an 80^3 27-point H (n = 640,000): its symbolic factor holds "
                                           "98 GB of L (lower triangles), 76 GB of it in one dense root front of "
                                           "order 137,520, and the root's three children hand it contribution "
                                           "blocks of order 126,472, 92,341 and 91,034 (64 + 34 + 33 GB, lower "
                                           "triangles): 229 GB together, and 151 GB for the root alone in this "
                                           "build's full m x k front panels: beyond one B200's 180 GB"}
        line["configs"] = side
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
