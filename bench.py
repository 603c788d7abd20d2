"""Benchmark of the B200 linear-solve path on the 24^3 P2 Euler-sized workload.

One step = one Newton linear solve: the block-ILU0 factorisation of a freshly
assembled Jacobian followed by FGMRES(50) to a relative residual of 1e-8 and
the true-residual check, all in FP64 (the plain GPU path).  Workload: 24x24x24
hex box, 5 fields, P2 (27 modes) -> 13 824 elements, 93 312 blocks of
135 x 135, 13.6 GB of FP64 blocks: the first Newton step's system of the
Euler equations on that box (freestream M 0.3 with a seeded Gaussian density
bump, farfield boundaries), its Jacobian assembled on the device by the DG
restatement, the pseudo-transient term at cfl 10 added, b = -R(q0).

Prints one JSON line (rank 0).  `value` times the solves with A and b resident
in HBM; `e2e` times the same solves through the C ABI from pinned host
buffers, host->device upload of A and b and download of x included in every
step, with two pipelines taking alternate steps so that one step's upload
overlaps the other's solve (`e2e.sequential`: one pipeline, no overlap).
`--impl reference` times the CPU FP64 oracle (the restatement of the
reference solver; the Fortran original cannot be built here) solving the same
24^3 system, one whole solve per step, on every host thread.  The GPU arm's
`cpu_baseline` is one such solve of its own headline system, which also gives
the GPU solution's relative error against the oracle (`rel_err_vs_oracle`).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton-Krylov solves/s + p50/p99 latency, mixed vs FP64 GPU at 1e-8 residual"
NX = NY = NZ = 24
P = 2
NVARS = 5
SEED_A, SEED_B = 1, 2
SOLVER = dict(tol=0.0, rtol=1e-8, nkrylov=50, inner_fgmres=0, nmax=500, orthogonalization="CGS",
              use_controller=0)
MIXED = dict(nkrylov=10, mixed_inner_nkrylov=30, mixed_inner_rtol=1e-2, mixed_inner_nmax=60)


def workload_config(extra=None):
    cfg = {"workload": "24^3 hex box, 5 fields, P2 (135x135 blocks, 93312 blocks, 13.6 GB FP64), "
                       "block-ILU0 factorisation + FGMRES(50) to rtol 1e-8, CGS, no inner FGMRES",
           "elements": NX * NY * NZ, "block": NVARS * (P + 1) ** 3, "blocks": 93312,
           "matrix_bytes_fp64": 13604889600, "l2_flush": "inputs larger than L2 (13.6 GB matrix)",
           "parallelism": "replicas",
           "values": "Euler DG Newton system at the initial state: Jacobian (assembled on the device) + the "
                     "pseudo-transient term at cfl 10, b = -R(q0); freestream M 0.3, rho 1, p 1/gamma, Gaussian "
                     "density bump (amplitude 1e-2, width 0.1, seeded centre in [0.3, 0.7]^3), farfield on every face"}
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# algorithmic work
# ---------------------------------------------------------------------------
def counts(pat):
    b = int(pat.bsize()[0])
    E = pat.nelem
    local = pat.blk_kind == 0
    nL = int((local & (pat.blk_col_elem < pat.blk_row_elem)).sum())
    nU = int((local & (pat.blk_col_elem > pat.blk_row_elem)).sum())
    NB = pat.nblocks
    return b, E, nL, nU, NB


def matvec_bytes(pat, sA=8, sv=8):
    b, E, nL, nU, NB = counts(pat)
    return NB * b * b * sA + (NB + E) * b * sv


def ilu_forward_bytes(pat, sL=8, sv=8):
    """L blocks read, v read, z written."""
    b, E, nL, nU, NB = counts(pat)
    return nL * b * b * sL + 2 * E * b * sv


def ilu_backward_bytes(pat, sL=8, sA=8, sv=8):
    """U blocks (from A) and inv(D) read, z read and written."""
    b, E, nL, nU, NB = counts(pat)
    return nU * b * b * sA + E * b * b * sL + 2 * E * b * sv


def fused_matvec_bytes(pat, sA=8, sv=8, sp=8):
    """The matvec rows inside the backward sweep: with the sweep's U partials
    reused (CHIDG_FUSED_REUSE, on by default), the diagonal and lower blocks
    and their x segments are read, the U partials (sp bytes a value) added,
    y written; otherwise the whole matvec."""
    if os.environ.get("CHIDG_FUSED_REUSE", "1").startswith("0"):
        return matvec_bytes(pat, sA, sv)
    b, E, nL, nU, NB = counts(pat)
    return (NB - nU) * b * b * sA + (NB - nU + E) * b * sv + nU * b * sp


def factor_flops(pat):
    b, E, nL, nU, NB = counts(pat)
    return 4 * nL * b ** 3 + 2 * E * b ** 3


# DRAM bytes of one launch (dram__bytes_read.sum + dram__bytes_write.sum)
# from ncu captures of the 14^3 P2 case (2744 elements, 18 032 blocks; the
# 24^3 workload is too large for a multi-pass capture), scaled to a launch of
# the workload by its block count.
TRAFFIC_14CUBE_BLOCKS = 18032
TRAFFIC_14CUBE = {"ilu_forward": 1.119160e9 + 14.508288e6, "ilu_backward": 1.520102e9 + 14.406656e6,
                  "ilu_backward_matvec": 3.051823e9 + 17.806592e6}


def measured_traffic(kind, pat):
    if kind not in TRAFFIC_14CUBE:
        return None
    if kind == "ilu_backward_matvec" and os.environ.get("CHIDG_FUSED_REUSE", "1").startswith("0"):
        return None           # the capture is of the matvec rows that reuse the U partials
    return TRAFFIC_14CUBE[kind] * pat.nblocks / TRAFFIC_14CUBE_BLOCKS


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------------------
# batched and served solves (independent systems of uneven size and order)
# ---------------------------------------------------------------------------
BATCH_SYSTEMS = 48
BATCH_OPTS = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=1000, use_controller=0)


_SYSTEMS = {}


def uneven_systems(count, seed, max_n=8, device=0):
    """Euler boxes with each side uniform in {4..max_n}, P uniform in {1, 2}
    (40x40 or 135x135 blocks), freestream Mach uniform in [0.2, 0.6] and bump
    amplitude uniform in [1e-3, 1e-2] (the scope table's draws for many solves,
    with smaller boxes): the first Newton step's system of each, assembled on
    the device and returned as host arrays (pattern, values, right-hand side)."""
    key = (count, seed, max_n)
    if key in _SYSTEMS:
        return _SYSTEMS[key]
    from chidg_b200 import api, euler
    ctx = api.default_context(device)
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(4, max_n + 1, size=3))
        P_ = int(rng.integers(1, 3))
        mach, amp = float(rng.uniform(0.2, 0.6)), float(rng.uniform(1e-3, 1e-2))
        centre = tuple(float(c) for c in rng.uniform(0.3, 0.7, 3))
        box = euler.EulerBox(nx, ny, nz, P_, vel_inf=(mach, 0.0, 0.0))
        q0 = box.density_bump(amplitude=amp, width=0.1, centre=centre)
        A = api.ChidgMatrix(box.pattern, ctx)
        b, _ = device_newton_system(ctx, A, box, q0)
        out.append((box.pattern, A.download(), b.download()))
        b.release()
        A.release()
    _SYSTEMS[key] = out
    return out


def run_batch_leg(ctx, schedule, reps=3):
    """The same systems solved one at a time (the plain FP64 path, and the
    FP32 inner solve) and batched (FP64, FP64 Krylov with FP32 preconditioner
    blocks, and FP64 outer steps preconditioned by batched FP32 inner solves);
    every mode to the same FP64 rtol 1e-8."""
    from chidg_b200 import api, mesh
    systems = uneven_systems(BATCH_SYSTEMS, seed=7)
    union, sys_elem = mesh.concat_patterns([s[0] for s in systems])
    A = api.ChidgMatrix(union, ctx)
    A.upload(np.concatenate([s[1] for s in systems]))
    b = api.ChidgVector(A, np.concatenate([s[2] for s in systems]))
    x = api.ChidgVector(A)
    M = api.create_preconditioner("ilu0", schedule=schedule)
    batched = {}
    for prec in ("fp64", "mixed_precon_fp32", "mixed_fp32"):
        solver = api.create_linear_solver("fgmres", **{**BATCH_OPTS, **(MIXED if prec == "mixed_fp32" else {})},
                                          precision=prec)
        solver.solve_batched(A, x, b, M, sys_elem)              # warm-up
        ctx.sync()
        t0 = time.perf_counter()
        for _ in range(reps):
            res = solver.solve_batched(A, x, b, M, sys_elem)
        ctx.sync()
        t = (time.perf_counter() - t0) / reps
        batched[prec] = {"solves_per_s": BATCH_SYSTEMS / t, "ms_per_batch": 1e3 * t,
                         "iterations": [r["niter"] for r in res],
                         "inner_iterations": [r["inner_iters"] for r in res],
                         "max_true_rel_residual": max(r["residual_norm"] / r["r0norm_initial"] for r in res)}
    M.tear_down()
    for o in (x, b, A):
        o.release()
    single = {"fp64": 0.0, "mixed_fp32": 0.0}
    for pat, vals, rhs in systems:
        As = api.ChidgMatrix(pat, ctx)
        As.upload(vals)
        bs, xs = api.ChidgVector(As, rhs), api.ChidgVector(As)
        Ms = api.create_preconditioner("ilu0", schedule=schedule)
        for prec in single:
            extra = dict(precision=prec, nkrylov=10, mixed_inner_nkrylov=30, mixed_inner_rtol=1e-2,
                         mixed_inner_nmax=60) if prec == "mixed_fp32" else {}
            opts = {**BATCH_OPTS, **extra}
            api.create_linear_solver("fgmres", **opts).solve(As, xs, bs, Ms)   # warm-up
            ctx.sync()
            t0 = time.perf_counter()
            api.create_linear_solver("fgmres", **opts).solve(As, xs, bs, Ms)
            ctx.sync()
            single[prec] += time.perf_counter() - t0
        Ms.tear_down()
        for o in (xs, bs, As):
            o.release()
    plain = BATCH_SYSTEMS / single["fp64"]
    return {"systems": BATCH_SYSTEMS,
            "workload": "boxes 4..8 per side, P in {1,2}, FGMRES(30)+ILU0 to rtol 1e-8 (FP64 residual)",
            "solves_per_s_one_at_a_time_fp64": plain,
            "solves_per_s_one_at_a_time_mixed_fp32": BATCH_SYSTEMS / single["mixed_fp32"],
            "solves_per_s_batched_fp64": batched["fp64"]["solves_per_s"],
            "solves_per_s_batched_mixed_precon_fp32": batched["mixed_precon_fp32"]["solves_per_s"],
            "solves_per_s_batched_mixed_fp32": batched["mixed_fp32"]["solves_per_s"],
            "speedup_vs_plain_fp64": {"batched_fp64": batched["fp64"]["solves_per_s"] / plain,
                                      "batched_mixed_precon_fp32": batched["mixed_precon_fp32"]["solves_per_s"] / plain,
                                      "batched_mixed_fp32": batched["mixed_fp32"]["solves_per_s"] / plain,
                                      "one_at_a_time_mixed_fp32": BATCH_SYSTEMS / single["mixed_fp32"] / plain},
            "batched": batched}


def run_serve_subprocess(device, timeout=900):
    """The serving leg in a fresh process on the same GPU: a request server is
    a process of its own, and its latencies must not depend on what the earlier
    legs left in this one (page-locked buffers, cached allocations, garbage)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--serve-only", "--serve-device", str(device)]
    # a server loads its kernels when it starts, not at a request's first use
    env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
    try:
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    except subprocess.TimeoutExpired:
        return {"error": "serving leg timed out"}
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    if p.returncode != 0 or not lines:
        return {"error": f"serving leg failed (exit {p.returncode}): {p.stderr.strip().splitlines()[-1:] }"}
    return json.loads(lines[-1])["serving"]


CFG5_REQUESTS = 512
CFG5_RATE = 200.0           # requests per second, Poisson
CFG5_SEED = 53
CFG5_BUDGET = 120 << 30     # device bytes the server admits at once (request_bytes estimates)
CFG5_SLOTS = 2
CFG5_MAX_BATCH = 32
CFG5_UNDER = (64, 4.0)      # a second stream below the GPU's capacity: requests, rate


def cfg5_requests(count=CFG5_REQUESTS, seed=CFG5_SEED):
    """The scope table's serving stream: systems drawn as the many-solve
    workload's (box sides uniform in 4..16, P in 1..3, Mach U[0.2, 0.6], bump
    amplitude U[1e-3, 1e-2]), every 10th request instead an Euler
    harmonic-balance system (8^3 P1, 3 harmonics: 7 coupled time levels, 280
    rows per element over the levels, sinusoidal inflow of amplitude 1e-2, the
    draw's Mach and bump).  Each request is the description of its first Newton
    step's system (euler.NewtonSystem); the server writes the system on the
    device when it admits the request (chidg_gpu_euler_fill_system), so no
    request's matrix is ever in host memory."""
    from chidg_b200 import euler, serve
    out = []
    for i, (shape, order, mach, amp, centre) in enumerate(cfg4_draws(count, seed)):
        if i % 10 == 9:
            sysm = euler.EulerHB(8, 8, 8, 1, [1.0, 2.0, 3.0], amplitude=1e-2, vel_inf=(mach, 0.0, 0.0))
        else:
            sysm = euler.EulerBox(*shape, order, vel_inf=(mach, 0.0, 0.0))
        desc = euler.NewtonSystem(sysm, sysm.density_bump(amplitude=amp, width=0.1, centre=centre), CFL_PTC)
        out.append(serve.SolveRequest(desc.pattern, None, None, tag=i, system=desc))
    return out


def batch_phases(log, t0):
    """Per-phase totals and maxima over a server's batch records (seconds), and
    the slowest batch's record with its times relative to the stream's start."""
    keys = [("queued", "formed", "taken"), ("on_device", "taken", "on_device"), ("set_up", "on_device", "set_up"),
            ("solve", "set_up", "solved"), ("to_host", "solved", "on_host")]
    out = {}
    for name, a, b in keys:
        d = [r[b] - r[a] for r in log]
        out[name] = {"sum_s": float(np.sum(d)), "max_s": float(np.max(d))} if d else None
    out["solve_device_s"] = float(np.sum([r["device_ms"] for r in log])) / 1e3 if log else None
    if log:
        worst = max(log, key=lambda r: r["on_host"] - r["taken"])
        out["slowest_batch"] = {k: (round(v - t0, 4) if k not in ("device_ms", "systems", "slot") else v)
                                for k, v in worst.items()}
    return out


def tune_for_serving(device):
    """The streamed kernels' shapes for the block-size classes of the served
    batches (largest block 40: P1 boxes and the harmonic-balance batches; 135;
    320: batches with P3 systems), in both precisions, measured by the project
    autotuner on arenas of each class.  The shape table is the process's, so
    the server's workers use them."""
    from chidg_b200 import api, tuning
    ctx = api.default_context(device)
    c = (0.5, 0.5, 0.5)
    arenas = ([((10, 10, 10), 1, 0.4, 5e-3, c)],
              [((8, 8, 8), 2, 0.4, 5e-3, c), ((10, 10, 10), 1, 0.3, 5e-3, c)],
              [((6, 6, 6), 3, 0.4, 5e-3, c), ((8, 8, 8), 2, 0.3, 5e-3, c), ((10, 10, 10), 1, 0.5, 5e-3, c)])
    shapes = {}
    t0 = time.perf_counter()
    for draws in arenas:
        A, b, _, _ = cfg4_arena(ctx, draws)
        for prec in ("mixed_fp32", "fp64"):
            M = api.create_preconditioner("ilu0")
            M.update(A, precision=prec)
            shapes.update(tuning.autotune(A, M, prec, reps=1))
            M.tear_down()
        b.release()
        A.release()
    ctx.sync()
    return shapes, time.perf_counter() - t0


def run_serve_leg(device, runs=1):
    """The serving configuration as stated: CFG5_REQUESTS requests arriving as
    a Poisson process at CFG5_RATE per second through the native server (two
    worker slots, admission by a device-memory budget), FGMRES(30) + ILU0 to
    rtol 1e-8 (FP64 residual), with FP32 inner solves (the mixed options of
    the single solves) and in plain FP64; then a shorter stream at a rate
    below the GPU's capacity.  Each run's batch records split the time into
    its phases."""
    from chidg_b200 import serve
    reqs = cfg5_requests()
    under = cfg5_requests(CFG5_UNDER[0], seed=CFG5_SEED + 1)
    # warm-up: the smallest request of each kind (order, time levels) among a few draws
    kinds = {}
    for r in cfg5_requests(40, seed=CFG5_SEED + 2):
        k = (int(r.pattern.elem_nterms[0]), r.pattern.ntime)
        if k not in kinds or r.pattern.nelem < kinds[k].pattern.nelem:
            kinds[k] = r
    warm = list(kinds.values())
    shapes, tune_s = tune_for_serving(device)
    import torch
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(min(CFG5_BUDGET, 0.75 * free))        # what the estimate may admit of the free memory
    out = {"workload": "Poisson arrivals of Euler Newton systems drawn as the many-solve workload (box sides 4..16, "
                       "P 1..3, Mach U[0.2, 0.6]), every 10th an Euler harmonic-balance system (8^3 P1, 7 levels); "
                       "each written on the device when admitted; FGMRES(30) + ILU0 to rtol 1e-8 (FP64 residual); "
                       "the server in a process of its own",
           "requests": len(reqs), "arrival_rate_per_s": CFG5_RATE, "slots": CFG5_SLOTS, "max_batch": CFG5_MAX_BATCH,
           "mem_budget_bytes": budget, "device_free_bytes_at_start": int(free),
           "server": "native (chidg_gpu_serve_*, chidg_gpu_serve_submit_fill)",
           "harmonic_balance_requests": sum(1 for r in reqs if r.pattern.ntime > 1),
           "matrix_bytes_fp64": int(sum(8 * r.pattern.value_offsets()[1] for r in reqs)),
           "below_capacity": {"requests": CFG5_UNDER[0], "arrival_rate_per_s": CFG5_UNDER[1]},
           "stream_shapes": shapes, "autotune_s": tune_s}

    def stream(prec, rq, rate, seed):
        srv = serve.NativeServer(device=device, slots=CFG5_SLOTS, max_batch=CFG5_MAX_BATCH, mem_budget=budget,
                                 **cfg4_opts(prec))
        try:
            for f in [srv.submit(r) for r in warm]:
                f.result()
            nwarm = srv.batches
            t0 = time.perf_counter()
            st = serve.run_stream(srv, rq, serve.poisson_arrivals(len(rq), rate, seed=seed))
            log = srv.batch_log()[nwarm:]
        finally:
            srv.close()
        res = st.pop("results")
        st["max_true_rel_residual"] = max(r.residual_norm / r.r0norm_initial for r in res)
        st["mean_iterations"] = float(np.mean([r.niter for r in res]))
        st["batches"] = len(log)
        st["phases"] = batch_phases(log, t0)
        return st

    for prec in ("mixed_fp32", "fp64"):
        results = [stream(prec, reqs, CFG5_RATE, 5) for _ in range(runs)]
        out[prec] = results[0] if runs == 1 else {"runs": results}
        under_runs = [stream(prec, under, CFG5_UNDER[1], 6) for _ in range(runs)]
        out["below_capacity"][prec] = under_runs[0] if runs == 1 else {"runs": under_runs}
    first = (lambda v: v if "runs" not in v else v["runs"][0])
    out["speedup_mixed_vs_fp64"] = first(out["mixed_fp32"])["solves_per_s"] / first(out["fp64"])["solves_per_s"]
    return out


# ---------------------------------------------------------------------------
# CPU legs (oracle)
# ---------------------------------------------------------------------------
def run_adjoint_leg(ctx, stream, A, b, schedule, reps=3):
    """The adjoint solve on the same 24^3 P2 system: A%transposed set, FGMRES(50)
    + ILU0 of A^T to rtol 1e-8 in FP64.  Each timed solve starts from a fresh
    A^T (A's stamp bumped, so its values are transposed again), as a Newton
    step's adjoint would."""
    import torch

    from chidg_b200 import api
    L = ctx.L
    A.transposed = True
    x = api.ChidgVector(A)
    y = api.ChidgVector(A)
    M = api.create_preconditioner("ilu0", schedule=schedule)
    solver = api.create_linear_solver("fgmres", **SOLVER)
    solver.solve(A, x, b, M)                       # warm-up: builds A^T and its programme
    bump = lambda: ctx.check(L.chidg_gpu_matrix_upload_range(A.h, None, 0, 0), "stamp")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    api.chidg_mv(A, b, y)
    torch.cuda.synchronize()
    ev[0].record(stream)
    api.chidg_mv(A, b, y)                          # A^T current: product only
    ev[1].record(stream)
    bump()
    ev[2].record(stream)
    api.chidg_mv(A, b, y)                          # transposition + product
    ev[3].record(stream)
    torch.cuda.synchronize()
    transpose_ms = ev[2].elapsed_time(ev[3]) - ev[0].elapsed_time(ev[1])
    lat = []
    for _ in range(reps):
        bump()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.solve(A, x, b, M)
        e1.record(stream)
        lat.append((e0, e1))
    torch.cuda.synchronize()
    ms = [a.elapsed_time(bb) for a, bb in lat]
    out = {"workload": "adjoint of the 24^3 P2 system: A^T x = b, FGMRES(50) + ILU0 of A^T to rtol 1e-8, FP64, "
                       "A^T re-transposed before every solve",
           "solves_per_s": 1000.0 * reps / sum(ms), "ms_per_solve": sum(ms) / reps,
           "transpose_ms": transpose_ms, "transpose_gbs": 2 * 8 * A.nvalues / (transpose_ms / 1e3) / 1e9,
           "iterations": solver.niter, "true_rel_residual": solver.residual_norm / solver.r0norm_initial}
    M.tear_down()
    for o in (x, y):
        o.release()
    A.transposed = False
    return out


def run_hb_leg(ctx, stream, schedule, reps=3):
    """A harmonic-balance request of the serving leg (the Euler box of
    hb_system: 8^3 P1, 7 time levels, hb_blks coupling every pair of levels):
    FGMRES(30) to rtol 1e-8, FP64, with ILU0 per time level and with
    precon_HB (per-element inverse over all levels)."""
    import torch

    from chidg_b200 import api
    pat, vals, rhs = hb_system(9, 11)
    A = api.ChidgMatrix(pat, ctx)
    A.upload(vals)
    b = api.ChidgVector(A, rhs)
    out = {"workload": "8^3 hex box, Euler under harmonic balance, P1, 3 harmonics = 7 time levels (40x40 blocks, "
                       "280x280 element blocks over the levels), sinusoidal inflow amplitude 1e-2, the first Newton "
                       "step's system; FGMRES(30) to rtol 1e-8, FP64"}
    for kind in ("ilu0", "hb"):
        M = api.create_preconditioner(kind, schedule=schedule)
        solver = api.create_linear_solver("fgmres", **{**SOLVER, "nkrylov": 30})
        x = api.ChidgVector(A)
        solver.solve(A, x, b, M)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            solver.solve(A, x, b, M)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[kind] = {"solves_per_s": 1000.0 / ms, "ms_per_solve": ms, "iterations": solver.niter,
                     "true_rel_residual": solver.residual_norm / solver.r0norm_initial}
        M.tear_down()
        x.release()
    b.release()
    A.release()
    return out


def run_newton_leg(ctx):
    """Whole Newton solve of five steps on cfg1: the 8^3 P1 box of the Euler
    equations (farfield on every face, freestream M = 0.3, rho = 1, p = 1/gamma,
    a Gaussian density bump of amplitude 1e-2 and width 0.1 at a seeded centre
    in [0.3, 0.7]^3), residual and Jacobian assembled on the host by the DG
    restatement, the Newton driver (pseudo-transient continuation from cfl 10,
    backtracking) over the device containers, each step's linear solve
    FGMRES(30) + ILU0 to rtol 1e-8 in FP64."""
    from chidg_b200 import api, euler
    from chidg_b200.newton import Newton
    rng = np.random.default_rng(SEED_A + 11)
    centre = tuple(float(c) for c in rng.uniform(0.3, 0.7, 3))
    box = euler.EulerBox(8, 8, 8, 1)
    A = api.ChidgMatrix(box.pattern, ctx)
    out = {"workload": "cfg1: 8^3 hex box, Euler, P1 (40x40 blocks), farfield, M 0.3 with a Gaussian density bump "
                       "(amplitude 1e-2, width 0.1): 5 Newton steps, host DG assembly, PTC cfl0 10, backtracking, "
                       "FGMRES(30)+ILU0 to rtol 1e-8 per step, FP64",
           "bump_centre": centre}
    q0 = box.density_bump(amplitude=1e-2, width=0.1, centre=centre)
    dev = euler.EulerDeviceSystem(box, ctx)
    for name, make in (("host_assembly", lambda: euler.EulerSystem(box)), ("device_assembly", lambda: dev)):
        for rep in range(2):                          # the first run warms up
            sysm = make()
            sysm.assemble_seconds, sysm.nassemble = 0.0, 0
            q = api.ChidgVector(A, q0)
            solver = api.create_linear_solver("fgmres", **{**SOLVER, "nkrylov": 30})
            res = Newton(nmax=5, tol=0.0, rtol=0.0, cfl0=10.0).solve(sysm, q, A, solver,
                                                                    api.create_preconditioner("ilu0"))
            q.release()
        out[name] = {"seconds_whole_newton": res.seconds, "steps": res.niter,
                     "seconds_linear_solves": float(sum(res.linear_seconds)),
                     "seconds_assembly": sysm.assemble_seconds, "assemblies": sysm.nassemble,
                     "residual_history": [float(r) for r in res.residual_norm],
                     "linear_iterations": res.matrix_iterations,
                     "linear_true_rel_residual": [float(r) for r in res.linear_rel_residual], "alphas": res.alphas,
                     "phase_seconds": res.phase_seconds}
    dev.device.release()
    A.release()
    return out


def run_assembly_leg(ctx, stream, A, reps=3):
    """The Euler DG residual and Jacobian of the 24^3 P2 box assembled on the
    device (k_euler_assemble) into the 24^3 P2 matrix (its values are
    overwritten: the leg runs after every leg that reads them), then one whole
    Newton step on it (the second of two, the first builds the ILU programme):
    assembly, pseudo-transient term, FGMRES(50) + ILU0 to rtol 1e-8,
    backtracking.  Farfield on every face, M 0.3 with a Gaussian
    density bump (amplitude 1e-2, width 0.1).  Algorithmic work per element:
    the DIAG block 25 nt rows x [qv (3 + nt) + 6 qf (1 + nt)] FMAs, each
    interior-face block 25 nt x qf (1 + nt) FMAs; bytes: the blocks and rhs
    written once, q read once."""
    import torch

    from chidg_b200 import api, euler
    from chidg_b200.newton import Newton
    box = euler.EulerBox(24, 24, 24, 2)
    dev = euler.EulerDevice(box, ctx)
    q0 = box.density_bump(amplitude=1e-2, width=0.1, centre=(0.45, 0.55, 0.5))
    q, r = api.ChidgVector(A, q0), api.ChidgVector(A)
    dev.assemble(q, r, A)                            # warm-up
    dev.assemble(q, r)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps + 2)]
    for i in range(reps):
        ev[2 * i].record(stream)
        dev.assemble(q, r, A)
        ev[2 * i + 1].record(stream)
    ev[-2].record(stream)
    dev.assemble(q, r)
    ev[-1].record(stream)
    torch.cuda.synchronize()
    jac_ms = sum(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(reps)) / reps
    res_ms = ev[-2].elapsed_time(ev[-1])
    nt, n1 = box.nterms, euler.nnodes_1d(box.order)
    qv, qf = n1 ** 3, n1 ** 2
    nface = sum(box._interior_pairs(d)[0].size for d in range(3)) * 2
    fma = box.nelem * 25 * nt * (qv * (3 + nt) + 6 * qf * (1 + nt)) + nface * 25 * nt * qf * (1 + nt)
    nbytes = 8 * (A.nvalues + 2 * A.n)
    out = {"workload": "Euler DG residual + Jacobian of the 24^3 P2 box on the device (93312 blocks of 135x135, "
                       "13.6 GB written), farfield, M 0.3 with a density bump",
           "jacobian_ms": jac_ms, "residual_only_ms": res_ms,
           "gflops": 2.0 * fma / (jac_ms / 1e3) / 1e9, "flops_per_call": 2.0 * fma,
           "gbs_written": nbytes / (jac_ms / 1e3) / 1e9, "bytes_per_call": nbytes}
    sysm = euler.EulerDeviceSystem(box, ctx)
    sysm.device.release()
    sysm.device = dev
    solver = api.create_linear_solver("fgmres", **SOLVER)
    M = api.create_preconditioner("ilu0")
    for rep in range(2):                             # the first step builds the ILU programme
        sysm.assemble_seconds, sysm.nassemble = 0.0, 0
        t0 = time.perf_counter()
        res = Newton(nmax=1, tol=0.0, rtol=0.0, cfl0=10.0).solve(sysm, q, A, solver, M)
    out["newton_step"] = {"seconds": time.perf_counter() - t0, "seconds_linear_solve": res.linear_seconds[0],
                          "seconds_assembly": sysm.assemble_seconds, "assemblies": sysm.nassemble,
                          "linear_iterations": res.matrix_iterations[0],
                          "linear_true_rel_residual": res.linear_rel_residual[0],
                          "residual_history": [float(v) for v in res.residual_norm], "alpha": res.alphas[0],
                          "phase_seconds": res.phase_seconds}
    M.tear_down()
    for o in (q, r):
        o.release()
    dev.release()
    return out


CFG3 = (32, 32, 32)
CFG3_SUB = (4, 4, 4)
CFG3_SOLVER = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=600, orthogonalization="CGS",
                   use_controller=0)


def run_cfg3_leg(ctx, stream, schedule, reps=2):
    """32^3 P2 Euler (223 232 blocks of 135 x 135, 32.5 GB FP64; freestream Mach
    drawn from a seeded U[0.2, 0.6]), the first Newton step's system:
    FGMRES(30) to rtol 1e-8 with block-ILU0 in FP64, with FP32 factors and FP32 Krylov, with BF16
    factors and FP32 Krylov, and RAS+ILU0 over 4 x 4 x 4 box subdomains of 8^3
    elements (each subdomain plays one MPI rank) in FP64 and with FP32 inner
    solves.  Every mode reaches the same FP64 true residual."""
    import torch

    from chidg_b200 import api, mesh
    mach = float(np.random.default_rng(SEED_B + 3).uniform(0.2, 0.6))
    t0 = time.perf_counter()
    box, q0, centre = euler_box(CFG3[0], SEED_A + 3, mach=mach, subdomains=CFG3_SUB)
    A = api.ChidgMatrix(box.pattern, ctx)
    b, assembly_s = device_newton_system(ctx, A, box, q0)
    setup_s = time.perf_counter() - t0
    x_ref = None
    out = {}
    for kind, prec in (("ilu0", "fp64"), ("ilu0", "mixed_fp32"), ("ilu0", "mixed_bf16"),
                       ("rasilu0", "fp64"), ("rasilu0", "mixed_fp32")):
        M = api.create_preconditioner(kind, schedule=schedule)
        opts = {**CFG3_SOLVER, "precision": prec}
        if prec != "fp64":
            opts.update(MIXED)
        solver = api.create_linear_solver("fgmres", **opts)
        x = api.ChidgVector(A)
        solver.solve(A, x, b, M)                       # warm-up (builds the programme)
        torch.cuda.synchronize()
        ctx.set_profiling(True)
        ev = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            solver.solve(A, x, b, M)
            e1.record(stream)
            ev.append((e0, e1))
        torch.cuda.synchronize()
        kt = ctx.kernel_times()
        ctx.set_profiling(False)
        lat = [a.elapsed_time(bb) for a, bb in ev]
        xh = x.download()
        if x_ref is None:
            x_ref = xh
        fa_ms, fa_n = kt.get("factor", (0.0, 0))
        out[f"{kind}_{prec}"] = {
            "solves_per_s": 1000.0 * reps / sum(lat), "ms_per_solve": sum(lat) / reps,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "outer_iters": solver.niter, "inner_iters": solver.inner_iters,
            "true_rel_residual": solver.residual_norm / solver.r0norm_initial,
            "rel_err_vs_ilu0_fp64_solution": float(np.linalg.norm(xh - x_ref) / np.linalg.norm(x_ref)),
            "factor_ms": fa_ms / fa_n if fa_n else None}
        M.tear_down()
        x.release()
    base = out["ilu0_fp64"]["ms_per_solve"]
    for v in out.values():
        v["speedup_vs_ilu0_fp64"] = base / v["ms_per_solve"]
    free, total = torch.cuda.mem_get_info()
    b.release()
    A.release()
    return {"workload": "32^3 hex box, Euler, P2 (223232 blocks of 135x135, 32.5 GB FP64): the first Newton step's "
                        "system (device-assembled Jacobian + pseudo-transient term at cfl 10, b = -R(q0)), FGMRES(30) "
                        "to rtol 1e-8 (FP64 true residual); RAS over 4x4x4 subdomains of 8^3, 1-element overlap",
            "mach": mach, "bump_centre": [float(c) for c in centre], "device_assembly_s": assembly_s,
            "setup_s": setup_s, "device_bytes_in_use_at_end": int(total - free), "modes": out}


CFG4_SYSTEMS = 512
CFG4_SEED = 41
CFG4_OPTS = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=1000, use_controller=0)
CFG4_WAVE_BYTES = 45e9      # FP64 matrix bytes per wave (the wave's device footprint is about 2.5 times that)
CFG4_SAMPLE = 24            # systems solved one at a time by the plain FP64 path (every 21st draw)


def cfg4_draws(count=CFG4_SYSTEMS, seed=CFG4_SEED):
    """The scope table's many-solve workload: each box side uniform in
    {4..16}, P uniform in {1, 2, 3} (40, 135, 320-row blocks), freestream Mach
    uniform in [0.2, 0.6], bump amplitude uniform in [1e-3, 1e-2], bump centre
    uniform in [0.3, 0.7]^3 (width 0.1)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        shape = tuple(int(v) for v in rng.integers(4, 17, size=3))
        P_ = int(rng.integers(1, 4))
        mach, amp = float(rng.uniform(0.2, 0.6)), float(rng.uniform(1e-3, 1e-2))
        centre = tuple(float(c) for c in rng.uniform(0.3, 0.7, 3))
        out.append((shape, P_, mach, amp, centre))
    return out


def box_matrix_bytes(shape, order):
    nx, ny, nz = shape
    b = NVARS * (order + 1) ** 3
    nl = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1)
    return (nx * ny * nz + 2 * nl) * b * b * 8


def cfg4_waves(draws, wave_bytes=CFG4_WAVE_BYTES):
    """Consecutive draws grouped into waves of at most wave_bytes of FP64
    matrix values (memory admission)."""
    waves, cur, cur_b = [], [], 0
    for d in draws:
        nb = box_matrix_bytes(d[0], d[1])
        if cur and cur_b + nb > wave_bytes:
            waves.append(cur)
            cur, cur_b = [], 0
        cur.append(d)
        cur_b += nb
    if cur:
        waves.append(cur)
    return waves


def cfg4_arena(ctx, draws):
    """One wave's systems packed block-diagonally into one matrix, each
    system's first Newton step written on the device straight into its slice
    (chidg_gpu_euler_fill_system: dR/dq(q0) + the pseudo-transient term at cfl
    CFL_PTC, b = -R(q0)).  Returns (A, b, sys_elem, seconds)."""
    from chidg_b200 import api, euler, mesh
    descs = []
    for shape, order, mach, amp, centre in draws:
        bx = euler.EulerBox(*shape, order, vel_inf=(mach, 0.0, 0.0))
        descs.append(euler.NewtonSystem(bx, bx.density_bump(amplitude=amp, width=0.1, centre=centre), CFL_PTC))
    union, sys_elem = mesh.concat_patterns([d.pattern for d in descs])
    t0 = time.perf_counter()
    A = api.ChidgMatrix(union, ctx)
    rhs, work = api.ChidgVector(A), api.ChidgVector(A)
    for d, e0 in zip(descs, sys_elem[:-1]):
        d.fill(A, rhs, work, int(e0))
    ctx.sync()
    work.release()
    return A, rhs, sys_elem, time.perf_counter() - t0


def cfg4_opts(prec):
    """The many-solve options of a precision mode (the FP32 inner solves take
    the mixed restart lengths and inner tolerance of the single solves)."""
    return {**CFG4_OPTS, **(MIXED if prec in ("mixed_fp32", "mixed_bf16") else {}), "precision": prec}


def run_cfg4_leg(ctx, schedule):
    """The many-solve configuration as stated: 512 Euler Newton systems of
    uneven size and order in memory-admitted waves, each wave packed into one
    arena and solved by the batched FGMRES(30) + ILU0 to rtol 1e-8 (FP64
    residual), with FP32 inner solves, with FP32 preconditioner blocks and in
    plain FP64; a sample of the draws also solved one at a time by the plain
    FP64 path."""
    from chidg_b200 import api, tuning
    draws = cfg4_draws()
    waves = cfg4_waves(draws)
    out = {"workload": f"{CFG4_SYSTEMS} Euler Newton systems: box sides uniform in 4..16, P uniform in 1..3 "
                       "(40/135/320-row blocks), Mach U[0.2, 0.6], bump amplitude U[1e-3, 1e-2]; memory-admitted "
                       f"waves of at most {CFG4_WAVE_BYTES / 1e9:.0f} GB of FP64 blocks, each packed into one arena; "
                       "batched FGMRES(30) + ILU0 to rtol 1e-8 (FP64 true residual); factorisation inside the timed solve",
           "systems": len(draws), "waves": len(waves),
           "orders": {str(p): sum(1 for d in draws if d[1] == p) for p in (1, 2, 3)},
           "matrix_bytes_fp64": int(sum(box_matrix_bytes(d[0], d[1]) for d in draws))}
    modes = {"mixed_fp32": 0.0, "mixed_precon_fp32": 0.0, "fp64": 0.0}
    iters = {k: [] for k in modes}
    inner = {k: [] for k in modes}
    worst = {k: 0.0 for k in modes}
    assembly_s = 0.0
    tuned = {}
    for wave in waves:
        A, b, sys_elem, asm = cfg4_arena(ctx, wave)
        assembly_s += asm
        x = api.ChidgVector(A)
        for prec in modes:
            M = api.create_preconditioner("ilu0", schedule=schedule)
            solver = api.create_linear_solver("fgmres", **cfg4_opts(prec))
            if schedule == "stream":
                M.update(A, precision=prec)
                key = (int(A.pattern.bsize().max()), prec)
                if key not in tuned:
                    tuned[key] = tuning.autotune(A, M, prec, reps=1, cache=os.environ.get("CHIDG_TUNE_CACHE"))
            ctx.sync()
            t0 = time.perf_counter()
            res = solver.solve_batched(A, x, b, M, sys_elem)
            ctx.sync()
            modes[prec] += time.perf_counter() - t0
            iters[prec] += [r["niter"] for r in res]
            inner[prec] += [r["inner_iters"] for r in res]
            worst[prec] = max(worst[prec], max(r["residual_norm"] / r["r0norm_initial"] for r in res))
            M.tear_down()
        x.release()
        b.release()
        A.release()
    # the plain FP64 path, one system at a time, on a sample of the draws, and
    # the same sample batched (its own waves), for a comparison on equal work
    sample = draws[::max(1, len(draws) // CFG4_SAMPLE)][:CFG4_SAMPLE]
    sample_batched = {"mixed_fp32": 0.0, "mixed_precon_fp32": 0.0, "fp64": 0.0}
    for wave in cfg4_waves(sample):
        A, b, sys_elem, _ = cfg4_arena(ctx, wave)
        x = api.ChidgVector(A)
        for prec in sample_batched:
            M = api.create_preconditioner("ilu0", schedule=schedule)
            solver = api.create_linear_solver("fgmres", **cfg4_opts(prec))
            ctx.sync()
            t0 = time.perf_counter()
            solver.solve_batched(A, x, b, M, sys_elem)
            ctx.sync()
            sample_batched[prec] += time.perf_counter() - t0
            M.tear_down()
        for o in (x, b, A):
            o.release()
    one = {"seconds": 0.0, "iterations": []}
    for d in sample:
        A, b, sys_elem, _ = cfg4_arena(ctx, [d])
        x = api.ChidgVector(A)
        M = api.create_preconditioner("ilu0", schedule=schedule)
        solver = api.create_linear_solver("fgmres", **CFG4_OPTS)
        ctx.sync()
        t0 = time.perf_counter()
        solver.solve(A, x, b, M)
        ctx.sync()
        one["seconds"] += time.perf_counter() - t0
        one["iterations"].append(solver.niter)
        M.tear_down()
        for o in (x, b, A):
            o.release()
    n = len(draws)
    out["device_assembly_s"] = assembly_s
    for prec, secs in modes.items():
        out[f"batched_{prec}"] = {"solves_per_s": n / secs, "seconds": secs, "mean_iterations": float(np.mean(iters[prec])),
                                  "max_iterations": int(max(iters[prec])), "max_true_rel_residual": worst[prec]}
        if prec == "mixed_fp32":
            out[f"batched_{prec}"]["mean_inner_iterations"] = float(np.mean(inner[prec]))
    sample_bytes = sum(box_matrix_bytes(d[0], d[1]) for d in sample)
    out["one_at_a_time_fp64_sample"] = {
        "systems": len(sample), "seconds": one["seconds"], "solves_per_s": len(sample) / one["seconds"],
        "matrix_bytes_fp64": int(sample_bytes), "mean_iterations": float(np.mean(one["iterations"])),
        "batched_mixed_fp32_solves_per_s": len(sample) / sample_batched["mixed_fp32"],
        "batched_mixed_precon_fp32_solves_per_s": len(sample) / sample_batched["mixed_precon_fp32"],
        "batched_fp64_solves_per_s": len(sample) / sample_batched["fp64"],
        "speedup_batched_mixed_fp32_vs_one_at_a_time_fp64": one["seconds"] / sample_batched["mixed_fp32"],
        "speedup_batched_mixed_precon_fp32_vs_one_at_a_time_fp64": one["seconds"] / sample_batched["mixed_precon_fp32"],
        "note": "every 21st draw, solved one at a time and batched (the same systems)"}
    out["speedup_batched_mixed_fp32_vs_batched_fp64"] = modes["fp64"] / modes["mixed_fp32"]
    out["speedup_batched_mixed_precon_fp32_vs_batched_fp64"] = modes["fp64"] / modes["mixed_precon_fp32"]
    out["stream_shapes"] = {f"b<={k[0]}/{k[1]}": v for k, v in tuned.items()}
    return out


CFL_PTC = 10.0          # pseudo-transient cfl of the Newton systems solved


def euler_box(n, seed, order=P, mach=0.3, subdomains=(1, 1, 1)):
    """The Euler box of the scope table's configurations: n^3 elements on
    [0,1]^3, freestream Mach `mach` (rho 1, p 1/gamma, so c = 1), a Gaussian
    density bump of amplitude 1e-2 and width 0.1 at a seeded centre in
    [0.3, 0.7]^3, farfield on every face; returns the box and q0."""
    from chidg_b200 import euler
    centre = np.random.default_rng(seed).uniform(0.3, 0.7, 3)
    box = euler.EulerBox(n, n, n, order, vel_inf=(mach, 0.0, 0.0), subdomains=subdomains)
    return box, box.density_bump(amplitude=1e-2, width=0.1, centre=tuple(centre)), centre


def device_newton_system(ctx, A, box, q0):
    """The first Newton step's linear system, on the device: A = dR/dq(q0) +
    mass / dtau (cfl CFL_PTC), returns b = -R(q0) and the assembly time."""
    from chidg_b200 import api, euler
    dev = euler.EulerDevice(box, ctx)
    q = api.ChidgVector(A, q0)
    b = api.ChidgVector(A)
    t0 = time.perf_counter()
    dev.assemble(q, b, A)
    dtau = dev.pseudo_timestep(q, CFL_PTC)
    A.scale_diagonal(box.mass, np.repeat(1.0 / dtau.min(axis=1), NVARS))   # minval over the fields
    b.scale(-1.0)
    ctx.sync()
    dt = time.perf_counter() - t0
    q.release()
    dev.release()
    return b, dt


_HB_SYSTEMS = {}


def hb_system(i, seed):
    """The harmonic-balance request of the scope table's serving workload: the
    8^3 P1 Euler box under harmonic balance with 3 harmonics (7 time levels,
    280 x 280 element blocks over the levels), a sinusoidal inflow of amplitude
    1e-2, a Gaussian density bump at a centre seeded by (request index, stream
    seed), so that streams of different seeds hold different systems; the
    first Newton step's system (pseudo-transient term at cfl 10), assembled on
    the device and cached as host arrays: (pattern, values, right-hand side)."""
    key = (i, seed)
    if key not in _HB_SYSTEMS:
        from chidg_b200 import api, euler
        centre = tuple(float(c) for c in np.random.default_rng((5000 + i, seed)).uniform(0.3, 0.7, 3))
        hb = euler.EulerHB(8, 8, 8, 1, [1.0, 2.0, 3.0], amplitude=1e-2)
        q0 = hb.density_bump(amplitude=1e-2, width=0.1, centre=centre)
        # assembled on the device (every level, the time coupling, the
        # pseudo-transient term of level 1 on every level's diagonal)
        ctx = api.default_context()
        A = api.ChidgMatrix(hb.pattern, ctx)
        q, r = api.ChidgVector(A, q0), api.ChidgVector(A)
        dev = euler.EulerHBDevice(hb, ctx)
        dev.assemble(q, r, A)
        dtau = dev.pseudo_timestep(q, A, CFL_PTC)
        A.scale_diagonal(hb.mass, np.repeat(1.0 / dtau.min(axis=1), NVARS))
        r.scale(-1.0)
        _HB_SYSTEMS[key] = (hb.pattern, A.download(), r.download())
        dev.release()
        for o in (q, r, A):
            o.release()
    return _HB_SYSTEMS[key]


def host_newton_system(n=NX, seed=SEED_A, order=P):
    """The workload's Newton system assembled on the host (the DG restatement
    in numpy): A = dR/dq(q0) + mass / dtau (cfl CFL_PTC, the element's smallest
    pseudo time step over its fields), b = -R(q0).  The same system as
    device_newton_system builds on the GPU."""
    from chidg_b200 import euler
    box, q0, _ = euler_box(n, seed, order=order)
    R, vals = box.residual(q0, jacobian=True)
    vals = euler.add_pseudo_time(box, vals, box.pseudo_timestep(q0, CFL_PTC))
    return box.pattern, vals, -R


def host_threads():
    return max(1, len(os.sched_getaffinity(0)))


def oracle_matrix(pat, vals):
    from oracle import oracle as O
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    return A


def oracle_solve(A, b, opts=None):
    """One full FGMRES(50)+ILU0 FP64 solve with the oracle (the restated
    reference solver), its ILU0 factorisation included (fgmres refreshes the
    preconditioner on every call without a controller, type_fgmres.f90:118-122),
    on the oracle's current host threads; returns (wall seconds, x, result)."""
    from oracle import oracle as O
    opts = {k: v for k, v in (opts or SOLVER).items() if k != "orthogonalization"}
    M = O.OraclePrecon(A, "ilu0")
    t0 = time.perf_counter()
    x, res = O.fgmres(A, M, b, O.default_opts(**opts))
    return time.perf_counter() - t0, x, res


def run_reference(args):
    """The reference's CPU solver on this host: the oracle's FGMRES(50) + block
    ILU0 (the restatement of type_fgmres.f90 and precon_ILU0.f90) solving the
    24^3 P2 Newton system itself, factorisation included, one whole solve per
    step, on every host thread (rows of one dependency level, matrix rows and
    independent Gram-Schmidt dots run in parallel; each row's arithmetic is the
    serial reference's, so x is bitwise the one-thread x)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    threads = host_threads()
    O.set_threads(threads)
    t0 = time.perf_counter()
    pat, vals, b = host_newton_system()
    A = oracle_matrix(pat, vals)
    del vals
    setup_s = time.perf_counter() - t0
    # warm-up steps: the ILU0 factorisation alone, which touches A and the
    # factor storage the timed solves use (a whole solve adds nothing to it)
    for _ in range(args.warmup):
        O.OraclePrecon(A, "ilu0").update()
    walls, niters = [], []
    for _ in range(args.steps):
        dt, x, res = oracle_solve(A, b)
        walls.append(dt)
        niters.append(res["niter"])
    total = float(sum(walls))
    value = args.steps / total
    sample = (f"the 24^3 P2 Euler Newton system itself (host-assembled), one whole FGMRES(50)+ILU0 FP64 solve per step "
              f"(factorisation included, {niters[-1]} iterations, true relative residual "
              f"{res['residual_norm'] / res['r0norm_initial']:.2e}) on {threads} host threads")
    lat = sorted(1000.0 * w for w in walls)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config({"precision": "fp64", "fgmres_iterations": niters,
                                       "implementation": "CPU FP64 oracle (the restated reference solver), "
                                                         f"{threads} host threads",
                                       "host_setup_s": setup_s}),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_oracle_check(pat, vals, rhs, x_gpu, solver, mixed_x):
    """The headline system solved by the oracle on every host thread (one whole
    FGMRES(50)+ILU0 FP64 solve, factorisation included): the GPU solution's
    relative error against it, the iteration counts and residual histories of
    both, each mixed mode's error against it, and the solve's wall time as the
    CPU baseline."""
    from oracle import oracle as O
    threads = host_threads()
    O.set_threads(threads)
    t0 = time.perf_counter()
    A = oracle_matrix(pat, vals)
    setup_s = time.perf_counter() - t0
    dt, xo, res = oracle_solve(A, np.array(rhs, copy=True))
    nx = float(np.linalg.norm(xo))
    hist_g, hist_o = np.asarray(solver.hist), np.asarray(res["hist"])
    m = min(hist_g.size, hist_o.size)
    check = {"oracle": f"CPU FP64 oracle, FGMRES(50)+ILU0, {threads} host threads",
             "rel_err_vs_oracle": float(np.linalg.norm(x_gpu - xo) / nx),
             "gpu_iterations": int(solver.niter), "oracle_iterations": int(res["niter"]),
             "max_rel_history_diff": float(np.max(np.abs(hist_g[:m] - hist_o[:m]) / hist_o[:m])) if m else None,
             "oracle_true_rel_residual": res["residual_norm"] / res["r0norm_initial"],
             "oracle_solve_s": dt, "oracle_setup_s": setup_s,
             "mixed_rel_err_vs_oracle": {k: float(np.linalg.norm(v - xo) / nx) for k, v in mixed_x.items()}}
    cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads, "kind": "port",
           "sample": f"one whole FGMRES(50)+ILU0 FP64 solve of this 24^3 P2 system itself (factorisation included, "
                     f"{res['niter']} iterations) by the oracle on {threads} host threads, {dt:.1f} s"}
    del A
    return check, cpu


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
def run_gpu(args):
    import torch

    from chidg_b200 import api, mesh
    from chidg_b200.replicas import allmax, barrier, init_from_env
    rank, world, local, pg = init_from_env("nccl")
    torch.cuda.set_device(local)
    # the library launches on this stream and every CUDA event below is recorded
    # on it (torch's default stream has handle 0, for which the library would
    # create a stream of its own)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = api.Context(local, stream=stream.cuda_stream)
    L0 = ctx.L
    pat = mesh.box_pattern(NX, NY, NZ, NVARS, mesh.nterms_of_order(P))
    nval = pat.value_offsets()[1]
    n = pat.vector_size()

    # pinned host copies of the inputs (the e2e leg uploads these every step)
    hv = torch.empty(nval, dtype=torch.float64, pin_memory=True)
    hb = torch.empty(n, dtype=torch.float64, pin_memory=True)
    hx = torch.empty(n, dtype=torch.float64, pin_memory=True)
    # the first Newton step's system of the Euler box, assembled on the device
    # (each rank its own seeded bump); the host copies are what e2e uploads
    box, q0, centre = euler_box(NX, SEED_A + 1000 * rank)
    A = api.ChidgMatrix(box.pattern, ctx)
    b, assembly_s = device_newton_system(ctx, A, box, q0)
    ctx.check(L0.chidg_gpu_matrix_download(A.h, api._ptr(hv.numpy())), "download A")
    ctx.check(L0.chidg_gpu_vector_download(b.h, api._ptr(hb.numpy())), "download b")
    x = api.ChidgVector(A)
    M = api.create_preconditioner("ilu0", schedule=args.schedule)
    solver = api.create_linear_solver("fgmres", **SOLVER)
    L = ctx.L
    # the project autotuner picks the streamed kernels' launch shapes for this
    # block size (before the warm-up; not timed)
    tuned, tune_s = None, None
    if args.schedule == "stream" and not args.no_tune:
        from chidg_b200 import tuning
        M.update(A)
        t0 = time.perf_counter()
        tuned = tuning.autotune(A, M, "fp64", reps=2, cache=os.environ.get("CHIDG_TUNE_CACHE"))
        tune_s = time.perf_counter() - t0

    def solve():
        solver.solve(A, x, b, M)

    # warm-up
    for _ in range(args.warmup):
        solve()
    niters = []
    lat = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    clocks = ClockSampler(local)
    barrier(pg, local)
    torch.cuda.synchronize()
    launches0 = ctx.launches()
    ctx.set_profiling(True)
    clocks.start()
    ev[0].record(stream)
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solve()
        e1.record(stream)
        niters.append(solver.niter)
        lat.append((e0, e1))
    ev[1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    kt = ctx.kernel_times()
    ctx.set_profiling(False)
    launches = ctx.launches() - launches0
    barrier(pg, local)
    elapsed_ms = ev[0].elapsed_time(ev[1])
    lat_ms = [a.elapsed_time(bb) for a, bb in lat]
    elapsed_ms = allmax(pg, elapsed_ms, local)
    value = world * args.steps / (elapsed_ms / 1000.0)
    resid = solver.residual_norm / solver.r0norm_initial

    # ---- end to end through the C ABI from pinned host buffers ----
    # Every step uploads its A and b from pinned host memory, solves, and
    # downloads x.  Sequentially, one step's upload waits for the previous
    # solve.  Pipelined, two lanes (each a context on a stream of its own with
    # its own matrix, preconditioner and solver, driven by a host thread) take
    # alternate steps, so one lane's upload overlaps the other's solve; each
    # solve still follows its own upload, and every copy is inside the timed
    # region, which opens with an event both streams wait on and closes after
    # both.  Uploads take the host link in turn: started together, the two
    # lanes' uploads would share it and finish together, and the lanes would
    # then run in lock-step with nothing overlapped.
    link = threading.Lock()          # the host link: one lane uploads while the other solves

    def e2e_step(c, Am, bm, xm, Mm, sm, hxm):
        with link:
            c.check(L.chidg_gpu_matrix_upload(Am.h, api._ptr(hv.numpy())), "upload A")
            c.check(L.chidg_gpu_vector_upload(bm.h, api._ptr(hb.numpy())), "upload b")
        sm.solve(Am, xm, bm, Mm)
        c.check(L.chidg_gpu_vector_download(xm.h, api._ptr(hxm.numpy())), "download x")

    nb_seq = max(1, min(args.steps, 3))
    barrier(pg, local)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nb_seq):
        e2e_step(ctx, A, b, x, M, solver, hx)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_seq_ms = allmax(pg, e0.elapsed_time(e1), local)
    e2e_seq_value = world * nb_seq / (e2e_seq_ms / 1000.0)

    stream2 = torch.cuda.Stream()
    ctx2 = api.Context(local, stream=stream2.cuda_stream)
    A2 = api.ChidgMatrix(box.pattern, ctx2)
    b2, x2 = api.ChidgVector(A2), api.ChidgVector(A2)
    M2 = api.create_preconditioner("ilu0", schedule=args.schedule)
    solver2 = api.create_linear_solver("fgmres", **SOLVER)
    hx2 = torch.empty(n, dtype=torch.float64, pin_memory=True)
    lanes = [(ctx, A, b, x, M, solver, hx), (ctx2, A2, b2, x2, M2, solver2, hx2)]
    e2e_step(*lanes[1])                                # the second lane's warm-up (its ILU programme)
    nb_e2e = 2 * max(1, min(args.steps, 4))
    errors = []

    def run_lane(i):
        try:
            for _ in range(i, nb_e2e, 2):
                e2e_step(*lanes[i])
        except Exception as exc:                     # re-raised on the main thread
            errors.append(exc)

    barrier(pg, local)
    torch.cuda.synchronize()
    p0, p1, p2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    p0.record(stream)
    stream2.wait_event(p0)
    lane_threads = [threading.Thread(target=run_lane, args=(i,)) for i in range(2)]
    for t in lane_threads:
        t.start()
    for t in lane_threads:
        t.join()
    if errors:
        raise errors[0]
    p2.record(stream2)
    stream.wait_event(p2)
    p1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = allmax(pg, p0.elapsed_time(p1), local)
    e2e_value = world * nb_e2e / (e2e_ms / 1000.0)
    e2e_x_agree = float(np.linalg.norm(hx2.numpy() - hx.numpy()) / max(np.linalg.norm(hx.numpy()), 1e-300))
    M2.tear_down()
    for o in (x2, b2, A2):
        o.release()
    ctx2.close()                                     # before its stream goes

    # ---- mixed precision (same workload, same 1e-8 target) ----
    mixed = {}
    mixed_x = {}
    if not args.no_mixed:
        for prec in ("mixed_precon_fp32", "mixed_fp32", "mixed_bf16"):
            # FP64 FGMRES(50) with FP32 preconditioner blocks; or an FP32 inner FGMRES
            opts = {**SOLVER, "precision": prec} if prec == "mixed_precon_fp32" else {**SOLVER, **MIXED, "precision": prec}
            ms = api.create_linear_solver("fgmres", **opts)
            xm = api.ChidgVector(A)
            if tuned is not None:                      # this precision's value widths get their own shapes
                from chidg_b200 import tuning
                M.update(A, precision=prec)
                tuning.autotune(A, M, prec, reps=2, cache=os.environ.get("CHIDG_TUNE_CACHE"))
            ms.solve(A, xm, b, M)                      # warm-up
            torch.cuda.synchronize()
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            nm = max(1, min(args.steps, 3))
            ctx.set_profiling(True)
            m0.record(stream)
            for _ in range(nm):
                ms.solve(A, xm, b, M)
            m1.record(stream)
            torch.cuda.synchronize()
            mkt = ctx.kernel_times()
            ctx.set_profiling(False)
            t = m0.elapsed_time(m1) / nm
            phases = {k: {"calls_per_solve": c / nm, "ms_per_call": (v / c if c else 0.0)}
                      for k, (v, c) in mkt.items() if c}
            xm_h = xm.download()
            x_h = x.download()
            mixed_x[prec] = xm_h
            mixed[prec] = {"solves_per_s": 1000.0 / t, "ms_per_solve": t, "outer_iters": ms.niter,
                           "inner_iters": ms.inner_iters,
                           "true_rel_residual": ms.residual_norm / ms.r0norm_initial,
                           "rel_err_vs_fp64_solution": float(np.linalg.norm(xm_h - x_h) / np.linalg.norm(x_h)),
                           "speedup_vs_fp64": (elapsed_ms / args.steps) / t, "phases": phases}
        M = api.create_preconditioner("ilu0", schedule=args.schedule)   # drop low-precision factors

    # ---- the oracle on the same system: parity of the headline solve and the CPU baseline ----
    oracle_check, cpu = None, None
    if not args.no_cpu and world == 1:
        oracle_check, cpu = run_oracle_check(box.pattern, hv.numpy(), hb.numpy(), x.download(), solver, mixed_x)
        for prec, err in oracle_check.pop("mixed_rel_err_vs_oracle").items():
            mixed[prec]["rel_err_vs_oracle"] = err

    # the single-GPU configurations' legs run in a one-GPU run only; a run of N
    # replicas measures the headline
    solo = world == 1
    adjoint = run_adjoint_leg(ctx, stream, A, b, args.schedule) if not args.no_adjoint and solo else None
    hb = run_hb_leg(ctx, stream, args.schedule) if not args.no_hb and solo else None
    newton = run_newton_leg(ctx) if not args.no_newton and solo else None
    batch = run_batch_leg(ctx, args.schedule) if not args.no_batch and solo else None
    assembly = run_assembly_leg(ctx, stream, A) if not args.no_assembly and solo else None
    cfg4 = run_cfg4_leg(ctx, args.schedule) if not args.no_cfg4 and solo else None
    # the 24^3 objects leave the device first: the 32^3 legs hold ~120 GB, the
    # serving process admits up to CFG5_BUDGET
    M.tear_down()
    for o in (x, b, A):
        o.release()
    ctx.sync()
    cfg3 = run_cfg3_leg(ctx, stream, args.schedule) if not args.no_cfg3 and solo else None
    # freed device memory leaves this process's pools at a synchronisation; the
    # serving process admits by what is free when it starts
    ctx.sync()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    serving = run_serve_subprocess(local) if not args.no_serve and solo else None

    if rank != 0:
        return 0

    hbm, bf16, peak_kind = measured_peaks()
    mv_ms, mv_n = kt["matvec"]
    f_ms, f_n = kt["ilu_forward"]
    bw_ms, bw_n = kt["ilu_backward"]
    bm_ms, bm_n = kt["ilu_backward_matvec"]
    fa_ms, fa_n = kt["factor"]
    mvb = matvec_bytes(pat)
    fwb, bwb = ilu_forward_bytes(pat), ilu_backward_bytes(pat)

    def cls(ms, cnt, nbytes):
        avg = ms / max(cnt, 1)
        return {"launches": cnt, "total_ms": ms, "avg_ms": avg, "algorithmic_bytes": nbytes,
                "gbs": nbytes / (avg / 1e3) / 1e9 if cnt else None}

    kernels = {
        "matvec": cls(mv_ms, mv_n, mvb),
        "ilu_forward": cls(f_ms, f_n, fwb),
        "ilu_backward": cls(bw_ms, bw_n, bwb),
        # the backward sweep with the following matvec's rows in the same launch
        "ilu_backward_matvec": cls(bm_ms, bm_n, bwb + fused_matvec_bytes(pat)),
        "factor": {"launches": fa_n, "total_ms": fa_ms, "avg_ms": fa_ms / max(fa_n, 1),
                   "tflops": factor_flops(pat) / (fa_ms / max(fa_n, 1) / 1e3) / 1e12 if fa_n else None},
    }
    # one Arnoldi step's z = M v and w = A z: forward sweep + (backward sweep and matvec)
    step_ms = kernels["ilu_forward"]["avg_ms"] + (kernels["ilu_backward_matvec"]["avg_ms"] if bm_n else
                                                  kernels["ilu_backward"]["avg_ms"] + kernels["matvec"]["avg_ms"])
    step_bytes = fwb + (bwb + fused_matvec_bytes(pat) if bm_n else bwb + mvb)
    kernels["precon_and_matvec_per_iteration"] = {"ms": step_ms, "algorithmic_bytes": step_bytes,
                                                  "gbs": step_bytes / (step_ms / 1e3) / 1e9}
    # dominant memory-bound kernel class by total time
    sweep = {"stream": "k_ilu_stream", "tasks": "k_ilu_tasks", "dataflow": "k_ilu_sweep_sf", "levels": "k_ilu_forward/backward"}
    names = {"matvec": "matvec (k_matvec_stream)", "ilu_forward": f"ilu_forward ({sweep[args.schedule]} forward)",
             "ilu_backward": f"ilu_backward ({sweep[args.schedule]} backward)",
             "ilu_backward_matvec": "ilu_backward_matvec (k_ilu_stream backward with the matvec rows)"}
    dom_key = max(names, key=lambda k: kernels[k]["total_ms"])
    dom, dbytes, dms = names[dom_key], kernels[dom_key]["algorithmic_bytes"], kernels[dom_key]["avg_ms"]
    achieved = dbytes / (dms / 1e3) / 1e9
    traffic = measured_traffic(dom_key, pat) if args.schedule == "stream" else None
    lat_sorted = sorted(lat_ms)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config({"precision": "fp64", "ilu_schedule": args.schedule, "fgmres_iterations": niters,
                                   "bump_centre": [float(c) for c in centre], "device_assembly_s": assembly_s,
                                   "true_rel_residual": resid, "stream_shapes": tuned, "autotune_s": tune_s,
                                   "rel_err_vs_oracle": oracle_check["rel_err_vs_oracle"] if oracle_check else None}),
        "oracle_check": oracle_check,
        "latency_ms": {"p50": float(np.percentile(lat_sorted, 50)), "p99": float(np.percentile(lat_sorted, 99))},
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(nval * 8 + n * 8),
                "d2h_bytes_per_step": int(n * 8), "steps": nb_e2e, "pipelines": 2,
                "sequential": {"value": e2e_seq_value, "steps": nb_seq}, "lanes_x_rel_diff": e2e_x_agree},
        "gpu_launches": launches,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dbytes},
        "kernels": kernels,
        "mixed": mixed,
        "batch": batch,
        "serving": serving,
        "adjoint": adjoint,
        "harmonic_balance": hb,
        "newton": newton,
        "euler_assembly": assembly,
        "cfg3": cfg3,
        "cfg4": cfg4,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--no-cpu", action="store_true",
                    help="skip the oracle solve of the headline system (cpu_baseline and rel_err_vs_oracle)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision legs")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-solve leg")
    ap.add_argument("--schedule", default="stream", choices=["tasks", "stream", "dataflow", "levels"],
                    help="schedule of the ILU sweeps")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (A^T) solve leg")
    ap.add_argument("--no-hb", action="store_true", help="skip the harmonic-balance preconditioner leg")
    ap.add_argument("--no-newton", action="store_true", help="skip the whole-Newton leg (8^3 P1, 5 steps)")
    ap.add_argument("--no-assembly", action="store_true",
                    help="skip the device Euler assembly leg (24^3 P2, overwrites the 24^3 matrix)")
    ap.add_argument("--no-cfg3", action="store_true", help="skip the 32^3 P2 legs (ILU0 and RAS, FP64 and mixed)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuning)")
    ap.add_argument("--no-cfg4", action="store_true",
                    help="skip the 512-system many-solve leg (sides 4..16, P 1..3, memory-admitted waves)")
    ap.add_argument("--serve-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--serve-device", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--serve-runs", type=int, default=1, help="streams per precision in the serving leg")
    args = ap.parse_args()
    if args.serve_only:
        import torch
        torch.cuda.set_device(args.serve_device)
        print(json.dumps({"serving": run_serve_leg(args.serve_device, runs=args.serve_runs)}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
