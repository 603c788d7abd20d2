"""A mid-size case of the hot kernels for profiler captures.

Runs `--reps` rounds of: ILU0 factorisation, one ILU0 apply (forward and
backward sweeps) and one FP64 matvec, on an n^3 P2 box (5 fields, 135 x 135
blocks).  n = 12 gives a 1.7 GB matrix: larger than L2 (126 MB), small enough
for multi-pass profiler captures.

  python -m chidg_b200.profile_case --n 12 --reps 2

With --euler: `--reps` device assemblies of the Euler DG residual and
Jacobian of the n^3 box at order p (farfield, M 0.3, a density bump) into the
box's matrix (k_euler_assemble).

With --fgmres k: `--reps` FGMRES(50) + ILU0 solves stopped after k iterations
(the factorisation, then per iteration the forward sweep and the backward
sweep with the matvec rows in one launch, k_ilu_stream with MV = true).
"""
from __future__ import annotations

import argparse

from . import api, mesh


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=12)
    ap.add_argument("--p", type=int, default=2)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--precon", default="ilu0")
    ap.add_argument("--schedule", default="stream", choices=["tasks", "stream", "dataflow", "levels"])
    ap.add_argument("--time", action="store_true", help="print CUDA-event times per kernel class")
    ap.add_argument("--solves", type=int, default=0, help="also time this many full solves per precision mode")
    ap.add_argument("--transposed", action="store_true", help="set A%%transposed (products and factors of A^T)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed_fp32", "mixed_bf16", "mixed_precon_fp32"],
                    help="precision of the preconditioner update (mixed_fp32 / mixed_bf16 factor in FP32 and skip "
                         "the FP64 apply)")
    ap.add_argument("--euler", action="store_true",
                    help="run the device Euler DG assembly (residual + Jacobian) instead of the solver kernels")
    ap.add_argument("--fgmres", type=int, default=0, help="run FGMRES solves of this many iterations instead")
    ap.add_argument("--tune", action="store_true", help="autotune the streamed kernels' shapes first (--fgmres)")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON file of tuned shapes: loaded when it holds this case's shapes, written otherwise")
    args = ap.parse_args()
    if args.euler:
        return euler_case(args)
    if args.fgmres:
        return fgmres_case(args)
    pat = mesh.box_pattern(args.n, args.n, args.n, 5, mesh.nterms_of_order(args.p))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=1))
    if args.transposed:
        A.transposed = True
    v = api.ChidgVector(A, mesh.synth_vector(A.n, seed=2))
    z = api.ChidgVector(A)
    M = api.create_preconditioner(args.precon, schedule=args.schedule)
    fp64_apply = args.precision in ("fp64", "mixed_precon_fp32")

    def round_():
        M.update(A, precision=args.precision)
        if fp64_apply:
            M.apply(A, v, z)
        api.chidg_mv(A, v, z)

    if args.time:
        # one untimed round first: launch set-up (function attributes,
        # occupancy queries) happens on the first call of each kernel
        round_()
        A.ctx.sync()
        A.ctx.set_profiling(True)
    for _ in range(args.reps):
        round_()
    A.ctx.sync()
    print(f"profile_case n={args.n} p={args.p} schedule={args.schedule}: {A.ctx.launches()} launches")
    if args.time:
        for name, (ms, cnt) in A.ctx.kernel_times().items():
            if cnt:
                print(f"  {name:14s} {cnt:4d} x {ms / cnt:9.3f} ms")
    if args.solves:
        solve_timings(args.n, args.p, args.solves, schedule=args.schedule)



def solve_timings(n=24, p=2, reps=6, precisions=("fp64", "mixed_fp32", "mixed_bf16"), schedule="stream"):
    """Wall time of full solves (factorisation + FGMRES) per precision mode."""
    import time
    pat = mesh.box_pattern(n, n, n, 5, mesh.nterms_of_order(p))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=1))
    b = api.ChidgVector(A, mesh.synth_vector(A.n, seed=2))
    x = api.ChidgVector(A)
    M = api.create_preconditioner("ilu0", schedule=schedule)
    out = {}
    for prec in precisions:
        opts = dict(tol=0.0, rtol=1e-8, nkrylov=50, inner_fgmres=0, nmax=500, precision=prec)
        if prec != "fp64":
            opts.update(nkrylov=10, mixed_inner_nkrylov=30, mixed_inner_rtol=1e-2, mixed_inner_nmax=60)
        s = api.create_linear_solver("fgmres", **opts)
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            s.solve(A, x, b, M)
            A.ctx.sync()
            times.append(time.perf_counter() - t0)
        out[prec] = (times, s.niter, s.inner_iters)
        print(f"  {prec:10s} iters {s.niter:3d}+{s.inner_iters:3d}  " + " ".join(f"{1e3 * t:7.1f}" for t in times) + " ms")
    return out


def fgmres_case(args):
    pat = mesh.box_pattern(args.n, args.n, args.n, 5, mesh.nterms_of_order(args.p))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=1))
    b = api.ChidgVector(A, mesh.synth_vector(A.n, seed=2))
    x = api.ChidgVector(A)
    M = api.create_preconditioner(args.precon, schedule=args.schedule)
    s = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-30, nkrylov=50, inner_fgmres=0, nmax=args.fgmres)
    if args.tune:
        from . import tuning
        M.update(A)
        print("shapes", tuning.autotune(A, M, "fp64", reps=2, cache=args.tune_cache))
    if args.time:
        s.solve(A, x, b, M)
        A.ctx.sync()
        A.ctx.set_profiling(True)
    for _ in range(args.reps):
        s.solve(A, x, b, M)
    A.ctx.sync()
    print(f"profile_case fgmres n={args.n} p={args.p}: {args.reps} solves of {s.niter} iterations, "
          f"{A.ctx.launches()} launches")
    if args.time:
        for name, (ms, cnt) in A.ctx.kernel_times().items():
            if cnt:
                print(f"  {name:20s} {cnt:4d} x {ms / cnt:9.3f} ms")


def euler_case(args):
    import time

    from . import euler
    box = euler.EulerBox(args.n, args.n, args.n, args.p)
    A = api.ChidgMatrix(box.pattern)
    dev = euler.EulerDevice(box, A.ctx)
    q = api.ChidgVector(A, box.density_bump(amplitude=1e-2, width=0.1, centre=(0.45, 0.55, 0.5)))
    r = api.ChidgVector(A)
    dev.assemble(q, r, A)
    A.ctx.sync()
    t0 = time.perf_counter()
    for _ in range(args.reps):
        dev.assemble(q, r, A)
    A.ctx.sync()
    ms = (time.perf_counter() - t0) * 1e3 / max(args.reps, 1)
    print(f"profile_case euler n={args.n} p={args.p}: {args.reps} assemblies, {ms:.3f} ms each (host clock), "
          f"{A.ctx.launches()} launches")


if __name__ == "__main__":
    main()
