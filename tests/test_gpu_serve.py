"""Continuous-batching server: requests of different sizes arriving while
others run are solved correctly, and each request's answer is the same
alone and in a mix (the batched solver never mixes systems' arithmetic)."""
import threading
import time

import numpy as np
import pytest

from chidg_b200 import _lib, api, euler, mesh, serve
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SIZES = [((3, 3, 2), 1), ((2, 2, 2), 2), ((4, 2, 2), 1), ((2, 2, 1), 0), ((3, 2, 2), 2), ((2, 3, 2), 1), ((3, 3, 3), 1)]
OPTS = dict(tol=0.0, rtol=1e-8, nkrylov=10, nmax=300)


def make_requests():
    reqs = []
    for i, (shape, P) in enumerate(SIZES):
        pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P))
        reqs.append(serve.SolveRequest(pat, mesh.synth_values(pat, seed=40 + i),
                                       mesh.synth_vector(pat.vector_size(), seed=80 + i), tag=i))
    return reqs


SERVERS = [serve.Server, serve.NativeServer]


@pytest.mark.parametrize("server", SERVERS)
def test_server_results_match_oracle_and_are_mix_independent(server):
    reqs = make_requests()
    srv = server(slots=2, max_batch=3, **OPTS)
    try:
        stats = serve.run_stream(srv, reqs, serve.poisson_arrivals(len(reqs), rate=200.0, seed=1))
        mixed = {r.tag: r for r in stats["results"]}
        alone = {}
        for req in make_requests():
            alone[req.tag] = srv.submit(req).result()
    finally:
        srv.close()
    assert stats["requests"] == len(reqs) and stats["p99_ms"] >= stats["p50_ms"] > 0
    for i, req in enumerate(make_requests()):
        Ao = O.OracleMatrix(req.pattern)
        Ao.set_values(req.values)
        xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), req.rhs, O.default_opts(inner_fgmres=0, **OPTS))
        assert mixed[i].niter == ro["niter"]
        assert np.linalg.norm(mixed[i].x - xo) <= 1e-10 * np.linalg.norm(xo)
        # same answer alone and in the mix
        assert np.array_equal(mixed[i].x, alone[i].x)


@pytest.mark.parametrize("server", SERVERS)
def test_server_admission_respects_memory_budget(server):
    reqs = make_requests()
    one = max(serve.request_bytes(r.pattern, OPTS["nkrylov"]) for r in reqs)
    srv = server(slots=3, max_batch=8, mem_budget=one, **OPTS)   # room for about one request at a time
    try:
        futs = [srv.submit(r) for r in reqs]
        res = [f.result(timeout=300) for f in futs]
    finally:
        srv.close()
    # admitted work never exceeded the budget, except a single batch larger than it
    assert srv.peak_mem_used <= one
    assert srv.batches >= 2
    assert all(r.residual_norm <= 2e-8 * r.r0norm_initial for r in res)


def fill_requests():
    out = []
    for i, (shape, P) in enumerate([((3, 2, 2), 1), ((2, 2, 2), 2), ((2, 3, 2), 1), ((2, 2, 2), 3)]):
        box = euler.EulerBox(*shape, P, vel_inf=(0.3 + 0.05 * i, 0.0, 0.0))
        q0 = box.density_bump(amplitude=0.02, width=0.3, centre=(0.5, 0.4, 0.5))
        out.append(serve.SolveRequest(box.pattern, None, None, tag=i, system=euler.NewtonSystem(box, q0, 10.0)))
    return out


@pytest.mark.parametrize("server", SERVERS)
def test_filled_requests_match_uploaded_ones(server):
    """Requests whose systems are written on the device when their batch is
    formed (chidg_gpu_serve_submit_fill with chidg_gpu_euler_fill_system) give
    bitwise the answers of the same systems handed over as host arrays, and
    every batch of the native server leaves a record of its phases."""
    reqs = fill_requests()
    uploaded = []
    for r in reqs:
        A = api.ChidgMatrix(r.pattern)
        b, w = api.ChidgVector(A), api.ChidgVector(A)
        r.system.fill(A, b, w, 0)
        uploaded.append(serve.SolveRequest(r.pattern, A.download(), b.download(), tag=r.tag))
        for o in (w, b, A):
            o.release()
    srv = server(slots=2, max_batch=3, **OPTS)
    try:
        filled = [f.result() for f in [srv.submit(r) for r in reqs]]
        up = [f.result() for f in [srv.submit(r) for r in uploaded]]
        log = srv.batch_log() if isinstance(srv, serve.NativeServer) else None
    finally:
        srv.close()
    for a, c in zip(filled, up):
        assert a.niter == c.niter and np.array_equal(a.x, c.x)
        assert a.residual_norm <= 2e-8 * a.r0norm_initial
    if log is not None:
        assert sum(r["systems"] for r in log) == 2 * len(reqs)
        for r in log:
            assert r["formed"] <= r["taken"] <= r["on_device"] <= r["set_up"] <= r["solved"] <= r["on_host"]
            assert r["device_ms"] > 0 and r["slot"] in (0, 1)


def test_native_server_splits_a_batch_that_runs_out_of_memory():
    """A batch whose systems do not fit on the device (here: a fill function
    that reports ENOMEM for every system but the first of a packed group) is
    solved in halves, in turn, down to single systems; every request still
    gets the answer it gets when uploaded."""
    reqs = fill_requests()[:3]
    blocker = fill_requests()[3]
    L = _lib.lib()
    seen = []
    gate = threading.Event()

    @_lib.FILL_FN
    def hold(user, ctx, A, b, work, elem0):
        gate.wait(60)                                 # keeps the only worker busy
        return L.chidg_gpu_euler_fill_system(user, ctx, A, b, work, elem0)

    @_lib.FILL_FN
    def tight(user, ctx, A, b, work, elem0):
        seen.append(elem0)
        if elem0 > 0:
            return _lib.ENOMEM
        return L.chidg_gpu_euler_fill_system(user, ctx, A, b, work, elem0)

    srv = serve.NativeServer(slots=1, max_batch=3, **OPTS)
    try:
        f0 = srv.submit_fill(blocker, hold, blocker.system.user, keep=blocker.system)
        time.sleep(0.5)
        futs = [srv.submit_fill(r, tight, r.system.user, keep=r.system) for r in reqs]
        gate.set()
        f0.result()
        got = [f.result() for f in futs]
        log = srv.batch_log()
        ref = [f.result() for f in [srv.submit(r) for r in fill_requests()[:3]]]
    finally:
        srv.close()
    assert any(r["systems"] == 3 for r in log)        # the three formed one batch
    assert any(e > 0 for e in seen)                   # which ran out and was split
    for a, c in zip(got, ref):
        assert a.niter == c.niter and np.array_equal(a.x, c.x)


def test_native_server_retries_a_system_alone_after_running_out_of_memory():
    """One system that runs out of device memory beside other batches (here:
    its fill function reports ENOMEM the first time) waits until it is the
    only batch on the device and is solved then."""
    req = fill_requests()[1]
    L = _lib.lib()
    calls = []

    @_lib.FILL_FN
    def once(user, ctx, A, b, work, elem0):
        calls.append(elem0)
        if len(calls) == 1:
            return _lib.ENOMEM
        return L.chidg_gpu_euler_fill_system(user, ctx, A, b, work, elem0)

    srv = serve.NativeServer(slots=2, max_batch=3, **OPTS)
    try:
        got = srv.submit_fill(req, once, req.system.user, keep=req.system).result(timeout=300)
        ref = srv.submit(fill_requests()[1]).result(timeout=300)
    finally:
        srv.close()
    assert len(calls) == 2
    assert got.niter == ref.niter and np.array_equal(got.x, ref.x)


def test_native_server_with_fp32_inner_solves():
    """The native server in the FP32-inner-solve mode: every request reaches
    the FP64 1e-8 residual, counts its inner iterations and agrees with its
    FP64 oracle solve."""
    reqs = make_requests()
    srv = serve.NativeServer(slots=2, max_batch=3, **OPTS, precision="mixed_fp32", mixed_inner_nkrylov=10,
                             mixed_inner_rtol=1e-2, mixed_inner_nmax=30)
    try:
        stats = serve.run_stream(srv, reqs, serve.poisson_arrivals(len(reqs), rate=200.0, seed=3))
    finally:
        srv.close()
    got = {r.tag: r for r in stats["results"]}
    for req in make_requests():
        r = got[req.tag]
        assert r.residual_norm <= 1.5e-8 * r.r0norm_initial, req.tag
        assert r.inner_iters >= r.niter > 0, req.tag
        Ao = O.OracleMatrix(req.pattern)
        Ao.set_values(req.values)
        xo, _ = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), req.rhs, O.default_opts(tol=0.0, rtol=1e-10, nkrylov=30,
                                                                                  inner_fgmres=0, nmax=300))
        assert np.linalg.norm(r.x - xo) <= 1e-6 * np.linalg.norm(xo), req.tag
