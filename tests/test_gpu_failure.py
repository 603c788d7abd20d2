"""Failure detection without a fault: the bounded device waits give up on a
flag nothing sets and an mbarrier nobody arrives at, report it, and leave
the context usable."""
import ctypes as C
import time

import numpy as np
import pytest

from chidg_b200 import api, mesh

pytestmark = pytest.mark.gpu


def test_bounded_waits_report_and_context_stays_usable():
    ctx = api.Context(0)
    bits = C.c_int32(-1)
    t0 = time.perf_counter()
    ctx.check(ctx.L.chidg_gpu_selftest_bounded_waits(ctx.h, 2_000_000, C.byref(bits)), "selftest")
    assert bits.value == 3                        # both waits gave up and said so
    assert time.perf_counter() - t0 < 10.0
    pat = mesh.box_pattern(2, 2, 1, 5, mesh.nterms_of_order(1))
    A = api.ChidgMatrix(pat, ctx)
    A.upload(mesh.synth_values(pat, seed=131))
    b = api.ChidgVector(A, mesh.synth_vector(pat.vector_size(), seed=132))
    x = api.ChidgVector(A)
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-8, nkrylov=20, inner_fgmres=0, nmax=100)
    solver.solve(A, x, b, api.create_preconditioner("ilu0"))
    assert solver.residual_norm <= 1.5e-8 * solver.r0norm_initial
