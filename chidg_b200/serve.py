"""Continuous-batching solve server.

Requests (one assembled Jacobian + right-hand side each) arrive at any time.
A dispatcher packs the waiting requests into batches, first come first
served, subject to a device-memory budget.  Each batch goes to a free worker
slot.  A slot owns its own context and CUDA stream, so batches that are
admitted while others are still on the GPU run concurrently with them.
Inside a batch the systems are solved together by
chidg_gpu_fgmres_solve_batched: one launch per matvec / ILU sweep /
reduction for all of them, and an independent Arnoldi process per system.
A system's arithmetic depends on the other systems of its batch only through
the launch shape of the batch's block-size class, so with one shape for every
class (the default) a request gets bitwise the same answer alone and in a mix.

Latency is measured from arrival to the result being back on the host.
"""
from __future__ import annotations

import collections
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

import ctypes as C

from . import _lib, api, mesh


@dataclass
class SolveRequest:
    """A system to solve: its assembled values and right-hand side in host
    memory, or (values and rhs None) `system`, an object with a `fill(A, b,
    work, elem0)` method that writes the system on the device when its batch
    is formed (euler.NewtonSystem: the native server then calls
    chidg_gpu_euler_fill_system itself)."""
    pattern: mesh.BlockPattern
    values: np.ndarray | None
    rhs: np.ndarray | None
    tag: object = None
    arrival: float = field(default_factory=time.perf_counter)
    system: object = None


@dataclass
class SolveResult:
    x: np.ndarray
    niter: int
    residual_norm: float
    r0norm_initial: float
    arrival: float
    start: float
    finish: float
    batch_size: int
    tag: object = None
    inner_iters: int = 0          # FP32 inner-solve iterations (mixed_fp32 / mixed_bf16)

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


def request_bytes(pat: mesh.BlockPattern, nkrylov: int, precision: str = "fp64") -> int:
    """Device bytes one request needs (an estimate for admission, as the
    native server makes it): its blocks, the ILU factors (the values of the
    diagonal and lower blocks in natural order), their FP32 copies in a mixed
    mode, the Krylov basis and a few vectors."""
    _, nval = pat.value_offsets()
    nr, nc = pat.block_dims()
    re, ce = np.asarray(pat.blk_row_elem), np.asarray(pat.blk_col_elem)
    rt, ct = np.asarray(pat.blk_row_time), np.asarray(pat.blk_col_time)
    low = (ce < re) | ((ce == re) & (ct <= rt))
    nlow = int((np.asarray(nr, dtype=np.int64) * np.asarray(nc, dtype=np.int64))[low].sum())
    n = pat.vector_size()
    blocks = 8 * (nval + nlow) + (4 * (nval + nlow) if precision != "fp64" else 0)
    return int(blocks + 8 * n * (2 * (nkrylov + 1) + 6))


class Server:
    """Continuous-batching server over `slots` concurrent GPU workers."""

    def __init__(self, device: int = 0, slots: int = 2, mem_budget: int = 60 << 30, max_batch: int = 32,
                 precon: str = "ilu0", **solver_options):
        self.device = device
        self.mem_budget = int(mem_budget)
        self.max_batch = max_batch
        self.precon = precon
        self.options = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=False, nmax=1000)
        self.options.update(solver_options)
        self._queue: "queue.Queue[tuple[SolveRequest, Future]]" = queue.Queue()
        self._free = threading.Semaphore(slots)
        self._mem_lock = threading.Condition()
        self._mem_used = 0
        self.peak_mem_used = 0
        self.batches = 0
        self._workers: list[threading.Thread] = []
        self._slot_ctx = queue.Queue()
        for _ in range(slots):
            self._slot_ctx.put(api.Context(device))
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._dispatcher.start()

    # -- public -------------------------------------------------------------
    def submit(self, req: SolveRequest) -> Future:
        fut: Future = Future()
        self._queue.put((req, fut))
        return fut

    def close(self):
        """Finish the queued requests, then stop the dispatcher and wait for the
        batches still on the GPU (no library call may outlive the server).  The
        slot contexts are released here: left to the garbage collector, their
        release (which frees device and page-locked memory, a device-wide
        synchronisation) could land in the middle of another server's work."""
        self._queue.put((None, None))
        self._dispatcher.join(timeout=600)
        for t in list(self._workers):
            t.join(timeout=600)
        while not self._slot_ctx.empty():
            self._slot_ctx.get_nowait().close()

    # -- internals ----------------------------------------------------------
    def _dispatch(self):
        pending = collections.deque()
        stopping = False

        def drain(block):
            nonlocal stopping
            while not stopping:
                try:
                    item = self._queue.get() if (block and not pending) else self._queue.get_nowait()
                except queue.Empty:
                    return
                if item[0] is None:
                    stopping = True
                    return
                pending.append(item)
                block = False

        while True:
            drain(block=True)
            if not pending:
                if stopping:
                    break
                continue
            self._free.acquire()                       # a worker slot is free
            drain(block=False)                         # requests that arrived meanwhile join
            # the oldest request, then the later ones of its number of time
            # levels that fit the memory not held by running batches, in arrival
            # order; requests passed over keep their place
            first = pending.popleft()
            batch = [first]
            nbytes = request_bytes(first[0].pattern, self.options["nkrylov"], self.options.get("precision", "fp64"))
            with self._mem_lock:
                room = self.mem_budget - self._mem_used
            keep = collections.deque()
            while pending:
                nxt = pending.popleft()
                need = request_bytes(nxt[0].pattern, self.options["nkrylov"], self.options.get("precision", "fp64"))
                if (len(batch) < self.max_batch and nbytes + need <= room
                        and nxt[0].pattern.ntime == first[0].pattern.ntime):
                    batch.append(nxt)
                    nbytes += need
                else:
                    keep.append(nxt)
            pending.extend(keep)
            with self._mem_lock:                        # admission by device memory
                while self._mem_used + nbytes > self.mem_budget and self._mem_used > 0:
                    self._mem_lock.wait()
                self._mem_used += nbytes
                self.peak_mem_used = max(self.peak_mem_used, self._mem_used)
                self.batches += 1
            ctx = self._slot_ctx.get()
            worker = threading.Thread(target=self._run_batch, args=(ctx, batch, nbytes), daemon=True)
            self._workers = [t for t in self._workers if t.is_alive()] + [worker]
            worker.start()

    def _run_batch(self, ctx, batch, nbytes):
        start = time.perf_counter()
        try:
            pats = [r.pattern for r, _ in batch]
            union, sys_elem = mesh.concat_patterns(pats)
            A = api.ChidgMatrix(union, ctx)
            b = api.ChidgVector(A)
            x = api.ChidgVector(A)
            eo = union.elem_offsets()
            v0 = o = 0
            for s, (r, _) in enumerate(batch):               # each request in place, no host copy
                n_s = int(eo[sys_elem[s + 1]] - eo[sys_elem[s]])
                nv_s = r.pattern.value_offsets()[1]
                if r.values is None:
                    r.system.fill(A, b, x, int(sys_elem[s]))
                else:
                    A.upload_range(np.ascontiguousarray(r.values, dtype=np.float64), v0)
                    b.upload_range(np.ascontiguousarray(r.rhs, dtype=np.float64), o)
                v0 += nv_s
                o += n_s
            x.clear()
            ctx.sync()
            M = api.create_preconditioner(self.precon)
            solver = api.create_linear_solver("fgmres", **self.options)
            res = solver.solve_batched(A, x, b, M, sys_elem)
            xh = x.download()
            finish = time.perf_counter()
            for s, (req, fut) in enumerate(batch):
                xs = xh[eo[sys_elem[s]]:eo[sys_elem[s + 1]]].copy()
                fut.set_result(SolveResult(xs, res[s]["niter"], res[s]["residual_norm"], res[s]["r0norm_initial"],
                                           req.arrival, start, finish, len(batch), req.tag, res[s]["inner_iters"]))
            M.tear_down()
            for o in (x, b, A):
                o.release()
        except Exception as exc:  # surface the failure on every request of the batch
            for _, fut in batch:
                if not fut.done():
                    fut.set_exception(exc)
        finally:
            with self._mem_lock:
                self._mem_used -= nbytes
                self._mem_lock.notify_all()
            self._slot_ctx.put(ctx)
            self._free.release()


class NativeServer:
    """The same continuous batching with the dispatcher and the worker slots as
    native threads behind the C ABI (chidg_gpu_serve_*), with the interface of
    Server.  A request's arrays are handed over by pointer: the returned
    future keeps them alive until its result has been taken."""

    def __init__(self, device: int = 0, slots: int = 2, mem_budget: int = 60 << 30, max_batch: int = 32,
                 precon: str = "ilu0", **solver_options):
        self.L = _lib.lib()
        self.options = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=False, nmax=1000)
        self.options.update(solver_options)
        self._solver = api.FGMRES(**self.options)       # the options struct of the batched solves
        h = C.c_void_p()
        self._t0 = time.perf_counter()                 # server timestamps count from its creation
        st = self.L.chidg_gpu_serve_create(int(device), int(slots), int(mem_budget), int(max_batch),
                                           api.PRECON_KINDS[precon.lower()], C.byref(self._solver._o), C.byref(h))
        if st:
            raise _lib.ChidgGpuError(st, "serve_create")
        self.h = h

    def submit(self, req: SolveRequest) -> "NativeFuture":
        if req.values is None:
            return self._submit_fill(req)
        values = np.ascontiguousarray(req.values, dtype=np.float64)
        rhs = np.ascontiguousarray(req.rhs, dtype=np.float64)
        pat = req.pattern.as_struct()
        ticket = C.c_int64()
        st = self.L.chidg_gpu_serve_submit(self.h, C.byref(pat), C.c_void_p(values.ctypes.data),
                                           C.c_void_p(rhs.ctypes.data), C.byref(ticket))
        if st:
            raise _lib.ChidgGpuError(st, "serve_submit")
        return NativeFuture(self, req, ticket.value, (values, rhs))

    def _submit_fill(self, req: SolveRequest) -> "NativeFuture":
        """chidg_gpu_serve_submit_fill with chidg_gpu_euler_fill_system and the
        request's euler.NewtonSystem as its description."""
        sysd = req.system
        if not hasattr(sysd, "user"):
            raise TypeError("the native server fills requests described by euler.NewtonSystem")
        return self.submit_fill(req, C.cast(self.L.chidg_gpu_euler_fill_system, C.c_void_p), sysd.user, keep=sysd)

    def submit_fill(self, req: SolveRequest, fill, user, keep=None) -> "NativeFuture":
        """chidg_gpu_serve_submit_fill with any chidg_gpu_fill_fn (a function
        address, or a _lib.FILL_FN callback) and its user pointer; `keep` (and
        the callback) stay referenced until the request's result is taken."""
        pat = req.pattern.as_struct()
        ticket = C.c_int64()
        fn = fill if isinstance(fill, C.c_void_p) else C.cast(fill, C.c_void_p)
        st = self.L.chidg_gpu_serve_submit_fill(self.h, C.byref(pat), fn, user, C.byref(ticket))
        if st:
            raise _lib.ChidgGpuError(st, "serve_submit_fill")
        return NativeFuture(self, req, ticket.value, (keep, fill))

    def batch_log(self) -> list[dict]:
        """The finished batches' records (chidg_gpu_serve_batch_log), times in
        seconds on the perf_counter clock of the requests' arrivals."""
        out = []
        rec = (C.c_double * 9)()
        for i in range(self.batches):
            if self.L.chidg_gpu_serve_batch_log(self.h, i, rec):
                continue
            t = [self._t0 + rec[k] for k in range(6)]
            out.append({"formed": t[0], "taken": t[1], "on_device": t[2], "set_up": t[3], "solved": t[4],
                        "on_host": t[5], "device_ms": rec[6], "systems": int(rec[7]), "slot": int(rec[8])})
        return out

    def _stats(self):
        if getattr(self, "h", None) is None:
            return self._final_stats                   # recorded by close()
        b, p = C.c_int64(), C.c_int64()
        self.L.chidg_gpu_serve_stats(self.h, C.byref(b), C.byref(p))
        return b.value, p.value

    @property
    def batches(self) -> int:
        return self._stats()[0]

    @property
    def peak_mem_used(self) -> int:
        return self._stats()[1]

    def close(self):
        """Solve everything queued, then stop the native threads."""
        if getattr(self, "h", None):
            self._final_stats = self._stats()
            self.L.chidg_gpu_serve_destroy(self.h)
            self.h = None


class NativeFuture:
    def __init__(self, server: NativeServer, req: SolveRequest, ticket: int, keep):
        self.server, self.req, self.ticket, self._keep = server, req, ticket, keep
        self._result = None

    def result(self, timeout=None) -> SolveResult:
        if self._result is None:
            x = np.empty(self.req.pattern.vector_size())
            res = _lib.FgmresResult()
            timing = (C.c_double * 4)()
            st = self.server.L.chidg_gpu_serve_wait(self.server.h, self.ticket, C.c_void_p(x.ctypes.data),
                                                    C.byref(res), timing)
            self._keep = None                          # the server no longer reads the request's arrays
            if st:
                raise _lib.ChidgGpuError(st, "serve_wait")
            t0 = self.server._t0
            self._result = SolveResult(x, res.niter, res.residual_norm, res.r0norm_initial, t0 + timing[0],
                                       t0 + timing[1], t0 + timing[2], int(timing[3]), self.req.tag, res.inner_iters)
        return self._result


def poisson_arrivals(n: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (s) of n requests of a Poisson process with the given rate."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def run_stream(server: Server, requests, arrivals) -> dict:
    """Submit requests at the given arrival times; return latency statistics."""
    t0 = time.perf_counter()
    futs = []
    for req, ta in zip(requests, arrivals):
        delay = t0 + ta - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        req.arrival = time.perf_counter()
        futs.append(server.submit(req))
    results = [f.result() for f in futs]
    t1 = max(r.finish for r in results)
    lat = np.array([r.latency for r in results])
    return {"requests": len(results), "wall_s": t1 - t0, "solves_per_s": len(results) / (t1 - t0),
            "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "mean_batch": float(np.mean([r.batch_size for r in results])), "results": results}
