"""Newton driver (newton_t%solve restated over the device containers) on a
synthetic nonlinear system with a known root, against the same loop run in
numpy with dense exact solves (residual history within 1e-6 relative: the
GPU's linear solves stop at rtol 1e-12)."""
import numpy as np
import pytest

from chidg_b200 import api, mesh
from chidg_b200.newton import Newton, NewtonOptions, SyntheticSystem

pytestmark = pytest.mark.gpu


def dense(pat, vals):
    n = pat.vector_size()
    D = np.zeros((n, n))
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    eo = pat.elem_offsets()
    b = pat.bsize()
    for k in range(pat.nblocks):
        r0 = eo[pat.blk_row_elem[k]] + pat.blk_row_time[k] * b[pat.blk_row_elem[k]]
        c0 = eo[pat.blk_col_elem[k]] + pat.blk_col_time[k] * b[pat.blk_col_elem[k]]
        D[r0:r0 + nr[k], c0:c0 + nc[k]] += vals[voff[k]:voff[k] + nr[k] * nc[k]].reshape(nc[k], nr[k]).T
    return D


def newton_numpy(sysm, q0, opts: NewtonOptions):
    """The driver's loop with dense matrices and exact solves."""
    A0 = dense(sysm.pattern, sysm.values0)
    block = int(sysm.pattern.bsize()[0])           # one element size throughout
    R = lambda q: A0 @ (q - sysm.qstar) + sysm.c * (q - sysm.qstar) ** 2
    q, hist, cfl, alphas = q0.copy(), [], opts.cfl0, []
    resid0 = np.linalg.norm(R(q))
    hist.append(resid0)
    for niter in range(1, 100):
        r = R(q)
        resid = np.linalg.norm(r)
        if resid < opts.tol:
            break
        J = A0 + 2 * sysm.c * np.diag(q - sysm.qstar)
        rhs = -r
        if opts.smooth and opts.ptc:
            # block Jacobi of J before the pseudo-transient term, on (M / dtau) r = r / cfl
            f = np.zeros_like(r)
            for i0 in range(0, len(q), block):
                f[i0:i0 + block] = np.linalg.solve(J[i0:i0 + block, i0:i0 + block], r[i0:i0 + block] / cfl)
            rhs = -r - opts.smooth_relax * f
        if opts.ptc:
            J = J + np.eye(len(q)) / cfl
        dq = np.linalg.solve(J, rhs)
        step = 0
        while True:
            alpha = 2.0 ** -step
            fn = np.linalg.norm(R(q + alpha * dq))
            step += 1
            if not ((fn > 1e-3 and fn > 2 * resid) or (fn < 1e-3 and fn > resid)):
                break
        q = q + alpha * dq
        alphas.append(alpha)
        cfl = cfl * (opts.cfl_up if alpha > 0.75 else (opts.cfl_down if alpha < 0.2 else 1.0))
        hist.append(fn)
        if not (fn > opts.tol and fn / resid0 > opts.rtol and (niter < opts.nmax or opts.nmax <= 0)):
            break
    return q, hist, alphas


@pytest.mark.parametrize("ptc,c,cfl0,smooth", [(True, 0.2, 100.0, False), (False, 0.2, 100.0, False),
                                                (True, 2.0, 1.0, False), (True, 0.2, 100.0, True),
                                                (True, 1.0, 5.0, True)])
def test_newton_matches_dense_loop(ptc, c, cfl0, smooth):
    """c = 2 from q0 = 0 takes backtracking steps (alpha < 1) and the cfl
    updates that follow them."""
    pat = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    sysm = SyntheticSystem(pat, seed=121, c=c, root_seed=122)
    A = api.ChidgMatrix(pat)
    q = api.ChidgVector(A)                           # q0 = 0
    opts = dict(tol=1e-9, rtol=1e-12, nmax=40, ptc=ptc, cfl0=cfl0, smooth=smooth, smooth_relax=0.5 if smooth else 1.0)
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=400)
    res = Newton(**opts).solve(sysm, q, A, solver, api.create_preconditioner("ilu0"))
    qn, hist, alphas = newton_numpy(sysm, np.zeros(pat.vector_size()), NewtonOptions(**opts))
    note = (res.residual_norm, hist, res.linear_rel_residual)
    assert max(res.linear_rel_residual) <= 1e-11, note          # every linear solve reached its tolerance
    # step by step while the iteration contracts slowly enough that 1e-12
    # differences in the linear solves stay below 1e-6 (the initial residual
    # and the first three steps);
    # a wandering iterate (c = 2) amplifies them later, so from there on both
    # runs need only converge to the same root
    m = min(len(hist), len(res.residual_norm), 4)
    for k in range(m):
        if hist[k] > 1e-6:
            assert abs(res.residual_norm[k] - hist[k]) <= 1e-6 * hist[k], (k, note)
    assert res.alphas[:4] == alphas[:4], note
    assert res.converged, note
    assert np.linalg.norm(qn - sysm.qstar) <= 1e-6 * np.linalg.norm(sysm.qstar)
    assert np.linalg.norm(q.download() - sysm.qstar) <= 1e-6 * np.linalg.norm(sysm.qstar)



def test_vector_mass_scale_matches_the_oracle():
    """chidg_gpu_vector_mass_scale (pseudo_transient_scaling) against the
    host restatement, on elements of two orders and three time levels."""
    from chidg_b200 import euler
    from oracle import newton_oracle
    for shape, P, T in (((3, 2, 2), 1, 1), ((2, 2, 1), 2, 3)):
        box = euler.EulerBox(*shape, P)
        pat = mesh.box_pattern(*shape, 5, box.nterms, ntime=T)
        A = api.ChidgMatrix(pat)
        x = api.ChidgVector(A, mesh.synth_vector(pat.vector_size(), seed=7))
        y = api.ChidgVector(A)
        dmin = np.linspace(0.5, 2.0, pat.nelem)
        y.assign_mass_scaled(x, box.mass, np.repeat(1.0 / dmin, 5))
        ref = newton_oracle.mass_scale(pat, x.download(), box.mass_block, dmin)
        assert np.abs(y.download() - ref).max() <= 1e-14 * np.abs(ref).max()
        with pytest.raises(api.ChidgGpuError):
            x.assign_mass_scaled(x, box.mass, np.repeat(1.0 / dmin, 5))


@pytest.mark.parametrize("smoother", ["jacobi", "preconditioner"])
def test_smoothed_newton_on_euler_matches_the_oracle_newton(smoother):
    """Residual smoothing (type_newton.f90:160-172) on the Euler box with the
    block-Jacobi smoother and with the linear solve's ILU0 as the smoother:
    the device loop's residual history within 1e-8 of the host restatement's."""
    from chidg_b200 import euler
    from oracle import newton_oracle
    from tests.test_gpu_config_parity import _HostEuler
    box = euler.EulerBox(4, 3, 3, 1, vel_inf=(0.3, 0.05, 0.0))
    q0 = box.density_bump(amplitude=2e-2, width=0.25, centre=(0.45, 0.5, 0.55))
    lin = dict(tol=0.0, rtol=1e-10, nkrylov=30, inner_fgmres=0, nmax=500)
    opts = dict(nmax=4, tol=0.0, rtol=0.0, cfl0=10.0, smooth=True, smoother=smoother, smooth_relax=0.7)
    A = api.ChidgMatrix(box.pattern)
    q = api.ChidgVector(A, q0)
    dev = euler.EulerDeviceSystem(box, A.ctx)
    res = Newton(**opts).solve(dev, q, A, api.create_linear_solver("fgmres", **lin), api.create_preconditioner("ilu0"))
    ref = newton_oracle.newton(_HostEuler(box), box.pattern, q0, linear_opts=lin, **opts)
    plain = newton_oracle.newton(_HostEuler(box), box.pattern, q0, linear_opts=lin,
                                 **{**opts, "smooth": False})
    note = (res.residual_norm, ref["residual_norm"])
    assert len(res.residual_norm) == len(ref["residual_norm"]) == 5, note
    for g, o in zip(res.residual_norm, ref["residual_norm"]):
        assert abs(g - o) <= 1e-8 * o, note
    assert res.alphas == ref["alphas"]
    assert ref["residual_norm"][1:] != plain["residual_norm"][1:]      # smoothing changed the steps
