"""The path on Euler DG Jacobians (chidg_b200.euler) instead of synthetic
values: the linear systems of a pseudo-transient Newton step solved by FGMRES +
ILU0 on the GPU against the oracle (pseudo-transient term added on the device
by scale_diagonal, on the host for the oracle), and whole Newton solves over
the device containers against a dense numpy Newton on the same host assembly.

Tolerances: FGMRES as the synthetic parity cases (same iteration count,
residual history within 1e-8 relative, solution within 1e-10 relative);
Newton residual history within 1e-6 relative while the iteration contracts
(the linear solves stop at rtol 1e-12, the dense one is exact)."""
import numpy as np
import pytest

from chidg_b200 import api, euler, mesh
from chidg_b200.newton import Newton, NewtonOptions
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def add_ptc(box, vals, dtau):
    """vals + mass / dtau on every field's diagonal sub-block of DIAG (host)."""
    nb, b, nt = box.pattern.nblocks, 5 * box.nterms, box.nterms
    out = vals.copy()
    blk = out.reshape(nb, b, b)                           # [block, column, row]
    for e in range(box.nelem):
        k = box._diag_k[e]
        for f in range(5):
            s = slice(f * nt, (f + 1) * nt)
            blk[k][s, s] += box.mass_block.T / dtau[e, f]
    return out


def dense(pat, vals):
    n = pat.vector_size()
    J = np.zeros((n, n))
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    eo = pat.elem_offsets()
    for k in range(pat.nblocks):
        r0, c0 = eo[pat.blk_row_elem[k]], eo[pat.blk_col_elem[k]]
        J[r0:r0 + nr[k], c0:c0 + nc[k]] += vals[voff[k]:voff[k] + nr[k] * nc[k]].reshape(nc[k], nr[k]).T
    return J


@pytest.mark.parametrize("shape,P,bcs", [((4, 3, 3), 1, "farfield"), ((3, 3, 2), 2, "farfield"),
                                         ((5, 2, 2), 1, ["farfield", "extrapolate"] * 3)])
@pytest.mark.parametrize("orth", ["CGS", "MGS"])
def test_newton_step_solve_parity(shape, P, bcs, orth):
    box = euler.EulerBox(*shape, P, bcs=bcs)
    q = box.density_bump(amplitude=1e-2, width=0.15, centre=(0.45, 0.55, 0.5))
    R, vals = box.residual(q, jacobian=True)
    dtau = box.pseudo_timestep(q, 10.0)
    Ao = O.OracleMatrix(box.pattern)
    Ao.set_values(add_ptc(box, vals, dtau))
    Ag = api.ChidgMatrix(box.pattern)
    Ag.upload(vals)
    Ag.scale_diagonal(box.mass, (1.0 / dtau).reshape(-1))
    assert relerr(Ag.download(), Ao.get_values()) < 1e-14
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=400, orthogonalization=orth)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), -R, O.default_opts(**opts))
    solver = api.create_linear_solver("fgmres", **opts)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, -R), api.create_preconditioner("ilu0"))
    assert solver.niter == ro["niter"]
    assert relerr(solver.hist, ro["hist"]) < 1e-8
    assert relerr(xg.download(), xo) < 1e-10


def newton_dense(box, q0, opts: NewtonOptions):
    """The driver's loop with dense matrices and exact solves, on the same
    host assembly."""
    M = np.zeros((q0.size, q0.size))
    nt = box.nterms
    for e in range(box.nelem):
        for f in range(5):
            s = (e * 5 + f) * nt
            M[s:s + nt, s:s + nt] = box.mass_block
    q, hist, alphas = q0.copy(), [], []
    cfl = np.full(5, opts.cfl0)
    resid0 = np.linalg.norm(box.residual(q))
    hist.append(resid0)
    for niter in range(1, 100):
        R, vals = box.residual(q, jacobian=True)
        resid = np.linalg.norm(R)
        J = dense(box.pattern, vals)
        if opts.ptc:
            J += M * (1.0 / box.pseudo_timestep(q, cfl)).reshape(-1).repeat(nt)[:, None]
        dq = np.linalg.solve(J, -R)
        step = 0
        while True:
            alpha = 2.0 ** -step
            fn = np.linalg.norm(box.residual(q + alpha * dq))
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


@pytest.mark.parametrize("shape,P,amp", [((4, 3, 3), 1, 1e-2), ((3, 3, 2), 2, 5e-2)])
def test_newton_on_euler_matches_dense(shape, P, amp):
    box = euler.EulerBox(*shape, P)
    sysm = euler.EulerSystem(box)
    q0 = box.density_bump(amplitude=amp, width=0.2, centre=(0.45, 0.55, 0.5))
    A = api.ChidgMatrix(box.pattern)
    q = api.ChidgVector(A, q0)
    opts = dict(tol=1e-12, rtol=1e-8, nmax=8, ptc=True, cfl0=10.0)
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=400)
    res = Newton(**opts).solve(sysm, q, A, solver, api.create_preconditioner("ilu0"))
    qd, hist, alphas = newton_dense(box, q0, NewtonOptions(**opts))
    note = (res.residual_norm, hist)
    assert max(res.linear_rel_residual) <= 1e-11, note
    assert len(res.residual_norm) == len(hist), note
    for a, b in zip(res.residual_norm, hist):
        assert abs(a - b) <= 1e-6 * b + 1e-15, note
    assert res.alphas == alphas
    assert hist[-1] < 1e-3 * hist[0]
    assert relerr(q.download(), qd) < 1e-8


DEVICE_CASES = [((3, 2, 2), 0, "farfield"), ((4, 3, 2), 1, "farfield"), ((3, 3, 2), 2, "farfield"),
                ((3, 2, 2), 1, ["farfield", "extrapolate"] * 3), ((2, 2, 3), 2, "extrapolate"), ((1, 1, 1), 1, "farfield"),
                ((3, 2, 2), 3, "farfield"), ((2, 2, 2), 3, ["extrapolate", "farfield"] * 3)]


@pytest.mark.parametrize("shape,P,bcs", DEVICE_CASES)
def test_device_assembly_matches_host(shape, P, bcs):
    """chidg_gpu_euler_assemble against the host restatement: residual within
    1e-12 of its norm, every Jacobian block within 1e-12 of the Jacobian's
    largest block (different summation order; each element integrates its own
    faces on the device)."""
    box = euler.EulerBox(*shape, P, bcs=bcs, vel_inf=(0.3, 0.1, -0.07), extent=((0, 1.2), (0, 1), (0, 0.9)))
    q = box.density_bump(amplitude=0.05, width=0.3, centre=(0.4, 0.5, 0.5))
    R, vals = box.residual(q, jacobian=True)
    dev = euler.EulerDevice(box)
    A = api.ChidgMatrix(box.pattern)
    qg, rg = api.ChidgVector(A, q), api.ChidgVector(A)
    dev.assemble(qg, rg, A)
    assert relerr(rg.download(), R) < 1e-12
    got = A.download()
    b = 5 * box.nterms
    scale = np.abs(vals).max()
    assert np.abs(got - vals).max() <= 1e-12 * scale
    assert np.abs(got - vals).reshape(-1, b * b).max(axis=1).max() <= 1e-12 * scale
    # residual only: same rhs, the matrix untouched
    stamp = A.stamp
    rg2 = api.ChidgVector(A)
    dev.assemble(qg, rg2)
    assert np.array_equal(rg2.download(), rg.download())
    assert A.stamp == stamp
    dtau = dev.pseudo_timestep(qg, [1.0, 2.0, 3.0, 4.0, 5.0])
    assert relerr(dtau, box.pseudo_timestep(q, [1.0, 2.0, 3.0, 4.0, 5.0])) < 1e-13


def test_device_assembly_rejects_other_patterns():
    box = euler.EulerBox(3, 2, 2, 1)
    dev = euler.EulerDevice(box)
    other = api.ChidgMatrix(euler.EulerBox(2, 3, 2, 1).pattern)      # same element count, other neighbours
    q, r = api.ChidgVector(other, box.freestream()), api.ChidgVector(other)
    with pytest.raises(RuntimeError):
        dev.assemble(q, r, other)
    small = api.ChidgMatrix(euler.EulerBox(2, 2, 2, 1).pattern)
    with pytest.raises(RuntimeError):
        dev.assemble(api.ChidgVector(small), api.ChidgVector(small))


def test_newton_device_assembly_matches_host_assembly():
    """The Newton driver with the assembly on the device against the same
    driver with the host assembly: the same steps, residuals within 1e-9."""
    box = euler.EulerBox(4, 3, 3, 1)
    q0 = box.density_bump(amplitude=1e-2, width=0.2, centre=(0.45, 0.55, 0.5))
    opts = dict(tol=1e-12, rtol=1e-8, nmax=6, ptc=True, cfl0=10.0)
    out = []
    for sysm in (euler.EulerSystem(box), euler.EulerDeviceSystem(box)):
        A = api.ChidgMatrix(box.pattern)
        q = api.ChidgVector(A, q0)
        solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=400)
        res = Newton(**opts).solve(sysm, q, A, solver, api.create_preconditioner("ilu0"))
        out.append((res, q.download()))
    (rh, qh), (rd, qd) = out
    assert len(rh.residual_norm) == len(rd.residual_norm)
    for a, b in zip(rd.residual_norm, rh.residual_norm):
        # relative 1e-9, with a floor of 1e-14 for the rounding of the O(1)
        # fluxes that sum to the last, small residuals (~1e-11 of |R0| here)
        assert abs(a - b) <= 1e-9 * b + 1e-14
    assert rd.alphas == rh.alphas
    assert relerr(qd, qh) < 1e-10


@pytest.mark.parametrize("kind", ["ilu0", "hb"])
def test_hb_newton_system_solve_parity(kind):
    """The harmonic-balance Euler system (euler.EulerHB: one harmonic, 3 time
    levels, a sinusoidal inflow; spatial blocks per level and D(t, t') mass
    hb blocks) with the pseudo-transient term: FGMRES with ILU0 per time level
    or precon_HB on the GPU against the oracle, the same bar as the steady
    systems."""
    hb = euler.EulerHB(3, 3, 2, 1, [1.0], amplitude=1e-2)
    q = hb.density_bump(amplitude=1e-2, width=0.15, centre=(0.45, 0.55, 0.5))
    R, vals = hb.residual(q, jacobian=True)
    vals = hb.add_pseudo_time(vals, hb.pseudo_timestep(q, 10.0))
    Ao = O.OracleMatrix(hb.pattern)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(hb.pattern)
    Ag.upload(vals)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=400)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, kind), -R, O.default_opts(**opts))
    solver = api.create_linear_solver("fgmres", **opts)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, -R), api.create_preconditioner(kind))
    assert solver.niter == ro["niter"]
    assert relerr(solver.hist, ro["hist"]) < 1e-8
    assert relerr(xg.download(), xo) < 1e-10


def test_assembly_into_a_batch_arena_matches_each_box():
    """Boxes of different sizes and orders assembled in place into their
    slices of one block-diagonal arena (chidg_gpu_euler_assemble_at): every
    slice is bitwise the box assembled alone, and the pseudo time steps too."""
    boxes = [euler.EulerBox(3, 2, 2, 1, vel_inf=(0.4, 0.0, 0.0)), euler.EulerBox(2, 2, 2, 3),
             euler.EulerBox(2, 3, 2, 2, vel_inf=(0.25, 0.05, 0.0))]
    qs = [bx.density_bump(amplitude=0.03, width=0.3, centre=(0.4, 0.5, 0.6)) for bx in boxes]
    union, sys_elem = mesh.concat_patterns([bx.pattern for bx in boxes])
    A = api.ChidgMatrix(union)
    q = api.ChidgVector(A, np.concatenate(qs))
    rhs = api.ChidgVector(A)
    dts = []
    for bx, e0 in zip(boxes, sys_elem[:-1]):
        dev = euler.EulerDevice(bx, A.ctx)
        dev.assemble_at(A, int(e0), q, rhs, True)
        dts.append(dev.pseudo_timestep_at(A, int(e0), q, 10.0))
        dev.release()
    vals, r = A.download(), rhs.download()
    voff, nval = union.value_offsets()
    eo = union.elem_offsets()
    first_blk = np.searchsorted(union.blk_row_elem, sys_elem[:-1])
    for s, (bx, qq) in enumerate(zip(boxes, qs)):
        Ab = api.ChidgMatrix(bx.pattern, A.ctx)
        qb, rb = api.ChidgVector(Ab, qq), api.ChidgVector(Ab)
        dev = euler.EulerDevice(bx, A.ctx)
        dev.assemble(qb, rb, Ab)
        v0 = voff[first_blk[s]]
        vb = Ab.download()
        assert np.array_equal(vals[v0:v0 + vb.size], vb), s
        assert np.array_equal(r[eo[sys_elem[s]]:eo[sys_elem[s]] + rb.n], rb.download()), s
        assert np.array_equal(dts[s], dev.pseudo_timestep(qb, 10.0)), s
        dev.release()


@pytest.mark.parametrize("order,freqs", [(1, [1.0, 2.0, 3.0]), (2, [1.5])])
def test_harmonic_balance_device_assembly_matches_host(order, freqs):
    """The harmonic-balance system assembled on the device (each level's
    spatial part by its own box, then the time coupling and the hb blocks)
    against the host EulerHB: residual within 1e-12 of its norm, every block
    within 1e-12 of the largest, the pseudo time steps of level 1 within 1e-13."""
    hb = euler.EulerHB(3, 2, 2, order, freqs, amplitude=2e-2, vel_inf=(0.35, 0.05, 0.0))
    q0 = hb.density_bump(amplitude=3e-2, width=0.3, centre=(0.4, 0.5, 0.5))
    R, vals = hb.residual(q0, jacobian=True)
    A = api.ChidgMatrix(hb.pattern)
    q, r = api.ChidgVector(A, q0), api.ChidgVector(A)
    dev = euler.EulerHBDevice(hb, A.ctx)
    dev.assemble(q, r, A)
    assert relerr(r.download(), R) < 1e-12
    got = A.download()
    assert np.abs(got - vals).max() <= 1e-12 * np.abs(vals).max()
    dt = dev.pseudo_timestep(q, A, 10.0)
    assert relerr(dt, hb.pseudo_timestep(q0, 10.0)) < 1e-13
    dev.release()


def host_driven_system(A, rhs, q, systems, sys_elem, cfl):
    """The Newton systems written the way the host drives it: assembly into
    each slice, dtau to the host, chidg_gpu_matrix_scale_diagonal over A with
    1 / min_f dtau, rhs = -rhs."""
    from chidg_b200 import _lib
    scale, mass = [], []
    for sysm, e0 in zip(systems, sys_elem[:-1]):
        if isinstance(sysm, euler.EulerHB):
            dev = euler.EulerHBDevice(sysm, A.ctx)
            L = A.ctx.L
            for t, lv in enumerate(dev.levels):
                A.ctx.check(L.chidg_gpu_euler_assemble_level_at(lv.h, A.h, int(e0), t, q.h, rhs.h, 1), "level_at")
            A.ctx.check(L.chidg_gpu_hb_coupling_at(A.h, int(e0), sysm.nelem, sysm.nterms, dev._D.ctypes.data_as(_lib.DP),
                                                   dev._M.ctypes.data_as(_lib.DP), q.h, rhs.h, 1), "hb_coupling_at")
            # level 1's dtau of this system, from a matrix of its own layout
            Ab = api.ChidgMatrix(sysm.pattern, A.ctx)
            eo = A.pattern.elem_offsets()
            qb = api.ChidgVector(Ab, q.download()[eo[e0]:eo[e0] + Ab.n])
            dt = dev.pseudo_timestep(qb, Ab, cfl)
            for o in (qb, Ab):
                o.release()
            dev.release()
        else:
            dev = euler.EulerDevice(sysm, A.ctx)
            dev.assemble_at(A, int(e0), q, rhs, True)
            dt = dev.pseudo_timestep_at(A, int(e0), q, cfl)
            dev.release()
        mass.append(sysm.mass)
        scale.append(np.repeat(1.0 / dt.min(axis=1), 5))
    A.scale_diagonal(np.concatenate(mass), np.concatenate(scale))
    rhs.scale(-1.0)


@pytest.mark.parametrize("kind", ["boxes", "hb"])
def test_fill_system_matches_host_driven_assembly(kind):
    """chidg_gpu_euler_fill_system (assembly, hb coupling, the pseudo-transient
    term and b = -R on the device, no host round trip) writes bitwise the
    system that the host-driven sequence writes, into each slice of a packed
    layout of several systems."""
    if kind == "boxes":
        systems = [euler.EulerBox(3, 2, 2, 1, vel_inf=(0.4, 0.0, 0.0)), euler.EulerBox(2, 2, 2, 3),
                   euler.EulerBox(2, 3, 2, 2, vel_inf=(0.25, 0.05, 0.0))]
    else:
        systems = [euler.EulerHB(2, 2, 2, 1, [1.0], amplitude=2e-2, vel_inf=(0.35, 0.05, 0.0)),
                   euler.EulerHB(3, 2, 1, 1, [1.5], amplitude=1e-2, vel_inf=(0.3, 0.0, 0.0))]
    qs = [s.density_bump(amplitude=0.03, width=0.3, centre=(0.4, 0.5, 0.6)) for s in systems]
    union, sys_elem = mesh.concat_patterns([s.pattern for s in systems])
    A1 = api.ChidgMatrix(union)
    q1, r1 = api.ChidgVector(A1, np.concatenate(qs)), api.ChidgVector(A1)
    host_driven_system(A1, r1, q1, systems, sys_elem, 10.0)
    A2 = api.ChidgMatrix(union, A1.ctx)
    b2, w2 = api.ChidgVector(A2), api.ChidgVector(A2)
    descs = [euler.NewtonSystem(s, qq, 10.0) for s, qq in zip(systems, qs)]
    for d, e0 in zip(descs, sys_elem[:-1]):
        d.fill(A2, b2, w2, int(e0))
    assert np.array_equal(A2.download(), A1.download())
    assert np.array_equal(b2.download(), r1.download())
    assert np.array_equal(w2.download(), np.concatenate(qs))   # work holds each q0
    for o in (q1, r1, A1, b2, w2, A2):
        o.release()


def test_fill_system_refuses_mismatched_layouts():
    box = euler.EulerBox(2, 2, 2, 1)
    d = euler.NewtonSystem(box, box.freestream(), 10.0)
    other = euler.EulerBox(2, 2, 2, 2)
    A = api.ChidgMatrix(other.pattern)
    b, w = api.ChidgVector(A), api.ChidgVector(A)
    with pytest.raises(api.ChidgGpuError):
        d.fill(A, b, w, 0)                       # modes differ
    Ab = api.ChidgMatrix(box.pattern, A.ctx)
    bb, wb = api.ChidgVector(Ab), api.ChidgVector(Ab)
    with pytest.raises(api.ChidgGpuError):
        d.fill(Ab, bb, wb, 1)                    # does not fit from element 1
    with pytest.raises(api.ChidgGpuError):
        d.fill(Ab, bb, bb, 0)                    # b and work must differ
    hb = euler.EulerHB(2, 2, 2, 1, [1.0])
    with pytest.raises(api.ChidgGpuError):
        euler.NewtonSystem(hb, hb.freestream(), 10.0).fill(Ab, bb, wb, 0)   # time levels differ
