"""Factor and solve one generated system: a command-line driver for timing and
profiling runs of the numeric phase.

    python rivrs-linalg_b200/run_step.py kkt 40 --precision mixed --reps 2
    python rivrs-linalg_b200/run_step.py lap 50 --precision fp64

`kkt G` is the saddle-point system on a G^3 27-point grid (n = 1.25 G^3),
`lap G` the 7-point Laplacian on a G^3 grid shifted to 5% negative
eigenvalues.  Each repetition is one factorization plus a solve refined to a
scaled backward error of 1e-14; the host wall time, refinement steps, backward
error and pivot counts are printed per repetition.
"""
import argparse
import os
import sys
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("kind", choices=["kkt", "lap"])
    ap.add_argument("grid", type=int)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--mixed-flush", type=int, default=4)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--no-scaling", action="store_true", help="skip MC64 scaling")
    ap.add_argument("--large-threshold", type=int, default=2048,
                    help="fronts of at least this order take the multi-kernel (whole GPU) path")
    ap.add_argument("--operands", default="tf32", choices=["tf32", "bf16"], help="mixed form: operand parts")
    ap.add_argument("--profile", action="store_true", help="print the factorization's time by kind of work")
    args = ap.parse_args()

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import __graft_entry__ as entry

    rv = entry.load_package()
    if args.kind == "kkt":
        s = rv.problems.kkt(args.grid, seed=0)
        b = rv.problems.rhs_normal(s.n, seed=0)
    else:
        s = rv.problems.shifted_laplacian(args.grid, 0.05)
        b = rv.problems.rhs_uniform(s.n, seed=0)
    if args.no_scaling:
        solver = rv.SparseLDLT.analyze(s)
    else:
        solver = rv.SparseLDLT.analyze_with_matrix(s, rv.AnalyzeOptions(rv.OrderingStrategy.MATCH_ORDER_METIS))
    opts = rv.FactorOptions(precision=args.precision, mixed_flush=args.mixed_flush,
                            large_front_threshold=args.large_threshold, mixed_operands=args.operands)
    if args.profile:
        solver._ensure_handle(opts)
        solver.set_profiling(True)
    for r in range(args.reps):
        t0 = time.perf_counter()
        solver.factor(s.values, opts)
        _, iters, err = solver.solve_refine(b, tol=1e-14, max_iter=10)
        print(f"rep {r}: n={s.n} {time.perf_counter() - t0:.3f} s refinement steps {iters} bwd err {err:.2e} "
              f"stats {solver.stats()}", flush=True)
        if args.profile:
            pr = solver.profile()
            print("  factor ms %.1f, parts %s" % (pr["factor_ms"], {k: round(v, 1) for k, v in pr["part_ms"].items()
                                                                 if v > 0}), flush=True)
    solver.close()


if __name__ == "__main__":
    main()
