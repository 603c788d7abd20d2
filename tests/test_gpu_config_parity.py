"""GPU parity at the sizes of the workload configurations, against the CPU
oracle on the same systems (the Euler Newton systems the bench solves):

cfg1  8^3 P1 Euler box, five Newton steps: the device path (device assembly,
      PTC through scale_diagonal, FGMRES(30) + ILU0 to rtol 1e-8) against the
      same Newton loop restated on the host (host assembly, the oracle's
      FGMRES + ILU0, oracle/newton_oracle.py): residual history within 1e-8
      relative, the same step lengths and linear iteration counts.
cfg2  24^3 P2 (13.6 GB FP64 blocks): one FGMRES(50) + ILU0 solve against one
      oracle solve of the same system: the same iteration count, residual
      history within 1e-8 relative, x within 1e-10 relative; every mixed
      precision mode reaches the FP64 1e-8 residual and lands within 1e-6 of
      the oracle's x.
cfg3  RAS + ILU0 over 4 x 4 x 4 box subdomains (16^3 P2, 4^3 elements each,
      one-element overlap): z = M v within 1e-11, and FGMRES(30) + RAS with
      the same iteration count, history within 1e-8 and x within 1e-10.

The oracle runs on every host thread (bitwise its one-thread results).
"""
import os

import numpy as np
import pytest

import bench
from chidg_b200 import api, euler
from chidg_b200.newton import Newton
from oracle import newton_oracle
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(autouse=True)
def _oracle_threads():
    O.set_threads(max(1, len(os.sched_getaffinity(0))))
    yield
    O.set_threads(1)


class _HostEuler:
    """The Euler box's residual, Jacobian and pseudo-transient term on the host."""

    def __init__(self, box):
        self.box = box

    def residual(self, q, jacobian=False):
        return self.box.residual(q, jacobian=jacobian)

    def pseudo_timestep(self, q, cfl):
        return self.box.pseudo_timestep(q, cfl)

    def add_pseudo_time(self, vals, dtau):
        return euler.add_pseudo_time(self.box, vals, dtau)

    @property
    def mass_block(self):
        return self.box.mass_block


def test_cfg1_newton_history_matches_the_oracle_newton():
    centre = tuple(float(c) for c in np.random.default_rng(bench.SEED_A + 11).uniform(0.3, 0.7, 3))
    box = euler.EulerBox(8, 8, 8, 1)
    q0 = box.density_bump(amplitude=1e-2, width=0.1, centre=centre)
    lin = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=500)
    newton = dict(nmax=5, tol=0.0, rtol=0.0, cfl0=10.0)
    A = api.ChidgMatrix(box.pattern)
    q = api.ChidgVector(A, q0)
    dev = euler.EulerDeviceSystem(box, A.ctx)
    res = Newton(**newton).solve(dev, q, A, api.create_linear_solver("fgmres", **lin),
                                 api.create_preconditioner("ilu0"))
    ref = newton_oracle.newton(_HostEuler(box), box.pattern, q0, **newton, linear_opts=lin)
    note = (res.residual_norm, ref["residual_norm"])
    assert res.niter == 5 and len(ref["residual_norm"]) == len(res.residual_norm) == 6, note
    for g, o in zip(res.residual_norm, ref["residual_norm"]):
        assert abs(g - o) <= 1e-8 * o, note
    assert res.alphas == ref["alphas"]
    assert res.matrix_iterations == ref["linear_iterations"]
    assert max(res.linear_rel_residual) <= 1e-8 * 1.0001
    assert relerr(q.download(), ref["q"]) <= 1e-9
    dev.device.release()


def _device_system(n, order, subdomains=(1, 1, 1), mach=0.3, seed=bench.SEED_A):
    box, q0, _ = bench.euler_box(n, seed, order=order, mach=mach, subdomains=subdomains)
    A = api.ChidgMatrix(box.pattern)
    b, _ = bench.device_newton_system(A.ctx, A, box, q0)
    return box, A, b


def test_cfg2_headline_solve_matches_an_oracle_solve():
    box, A, b = _device_system(24, 2)
    vals, rhs = A.download(), b.download()
    Ao = O.OracleMatrix(box.pattern)
    Ao.set_values(vals)
    del vals
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), rhs,
                      O.default_opts(**{k: v for k, v in bench.SOLVER.items() if k != "orthogonalization"}))
    del Ao
    M = api.create_preconditioner("ilu0")
    x = api.ChidgVector(A)
    solver = api.create_linear_solver("fgmres", **bench.SOLVER)
    solver.solve(A, x, b, M)
    assert solver.niter == ro["niter"]
    assert np.max(np.abs(solver.hist - ro["hist"]) / ro["hist"]) <= 1e-8
    assert relerr(x.download(), xo) <= 1e-10
    for prec in ("mixed_precon_fp32", "mixed_fp32", "mixed_bf16"):
        opts = {**bench.SOLVER, "precision": prec}
        if prec != "mixed_precon_fp32":
            opts.update(bench.MIXED)
        ms = api.create_linear_solver("fgmres", **opts)
        xm = api.ChidgVector(A)
        ms.solve(A, xm, b, M)
        assert ms.residual_norm / ms.r0norm_initial <= 1e-8 * 1.0001, prec
        assert relerr(xm.download(), xo) <= 1e-6, prec
        xm.release()
    M.tear_down()


def test_cfg3_ras_4x4x4_matches_the_oracle():
    box, A, b = _device_system(16, 2, subdomains=(4, 4, 4), mach=0.5)
    vals, rhs = A.download(), b.download()
    Ao = O.OracleMatrix(box.pattern)
    Ao.set_values(vals)
    Mo = O.OraclePrecon(Ao, "rasilu0")
    Mo.update()
    M = api.create_preconditioner("rasilu0")
    M.init(A)
    M.update(A)
    v = rhs / np.linalg.norm(rhs)
    z = M.apply(A, api.ChidgVector(A, v)).download()
    assert relerr(z, Mo.apply(v)) <= 1e-11
    opts = {**bench.CFG3_SOLVER}
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "rasilu0"), rhs,
                      O.default_opts(**{k: v for k, v in opts.items() if k != "orthogonalization"}))
    x = api.ChidgVector(A)
    solver = api.create_linear_solver("fgmres", **opts)
    solver.solve(A, x, b, M)
    assert solver.niter == ro["niter"]
    assert np.max(np.abs(solver.hist - ro["hist"]) / ro["hist"]) <= 1e-8
    assert relerr(x.download(), xo) <= 1e-10
    M.tear_down()
