"""Euler DG residual and Jacobian on hex boxes (chidg_b200.euler), on the CPU.

No reference output exists here to pin the assembly (the reference needs a
Fortran compiler, HDF5 and MPI), so it is held to the properties a correct DG
discretisation has: the mode order and basis of the reference, freestream
preservation, consistency and conservation of the face fluxes, a Jacobian equal
to the derivative of the residual, and exact projection of polynomials."""
import numpy as np
import pytest

from chidg_b200 import euler


def test_mode_order_shells():
    """Every prefix of (P+1)^3 modes is the full order-P tensor set, and the
    first modes are the reference's (mod_ordering.f90: 1; then (1,2,1), (1,1,2),
    (2,1,1), ... 1-based)."""
    for P in range(euler.MAX_ORDER + 1):
        n = (P + 1) ** 3
        got = sorted(map(tuple, euler.MODE_ORDER[:n]))
        assert got == sorted((a, b, c) for a in range(P + 1) for b in range(P + 1) for c in range(P + 1))
    assert list(map(tuple, euler.MODE_ORDER[:4])) == [(0, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 0)]


def test_legendre_tables_match_numpy():
    x = np.linspace(-1, 1, 17)
    L, D = euler._legendre_tables(5, x)
    for n in range(6):
        c = np.zeros(n + 1)
        c[n] = 1.0
        assert np.allclose(L[n], np.polynomial.legendre.legval(x, c), atol=1e-14)
        assert np.allclose(D[n], np.polynomial.legendre.legval(x, np.polynomial.legendre.legder(c)), atol=1e-13)


def test_quadrature_rule():
    assert [euler.nnodes_1d(P) for P in range(4)] == [2, 3, 5, 6]


@pytest.mark.parametrize("P", [0, 1, 2])
def test_mass_matrix_diagonal(P):
    b = euler.EulerBox(2, 3, 1, P, extent=((0, 2), (0, 1.5), (-1, 1)))
    deg = euler.MODE_ORDER[:b.nterms]
    want = b.vol * np.prod(1.0 / (2 * deg + 1), axis=1)
    assert np.allclose(b.mass_block, np.diag(want), atol=1e-15 * b.vol)


@pytest.mark.parametrize("bcs", ["farfield", "extrapolate"])
@pytest.mark.parametrize("P", [0, 1, 2])
def test_freestream_preserved(bcs, P):
    b = euler.EulerBox(3, 2, 2, P, bcs=bcs, vel_inf=(0.3, 0.1, -0.05), extent=((0, 1.5), (0, 1), (0, 0.8)))
    q = b.freestream()
    assert np.abs(b.residual(q)).max() < 1e-13


def test_projection_exact_for_polynomials():
    b = euler.EulerBox(2, 2, 2, 2)

    def fn(x):
        out = np.empty(x.shape[:-1] + (5,))
        out[..., 0] = 1.0 + 0.1 * x[..., 0] * x[..., 1] + 0.05 * x[..., 2] ** 2
        out[..., 1:4] = x[..., :3] ** 2
        out[..., 4] = 2.0 + x[..., 0] * x[..., 1] * x[..., 2]
        return out
    q = b.modes(b.project(fn))
    vals = np.einsum("qm,efm->eqf", b.phi, q)
    assert np.allclose(vals, fn(b.coords()), atol=1e-13)


def _states(rng, n):
    rho = 1.0 + 0.2 * rng.random(n)
    u = 0.3 * rng.standard_normal((n, 3))
    p = 0.7 + 0.2 * rng.random(n)
    Q = np.empty((n, 5))
    Q[:, 0] = rho
    Q[:, 1:4] = rho[:, None] * u
    Q[:, 4] = p / (euler.GAMMA - 1) + 0.5 * rho * (u * u).sum(1)
    return Q


def test_roe_flux_consistent_and_conservative():
    """The upwind term vanishes for equal states, and the numerical flux is
    antisymmetric: F(QL, QR, n) = -F(QR, QL, -n)."""
    rng = np.random.default_rng(3)
    QL, QR = _states(rng, 50), _states(rng, 50)
    n = np.array([0.6, -0.48, 0.64])
    assert np.abs(euler.roe_upwind(QL, QL, n)).max() < 1e-14
    fl = np.einsum("qdf,d->qf", 0.5 * (euler.euler_flux(QL) + euler.euler_flux(QR)), n) + euler.roe_upwind(QL, QR, n)
    fr = np.einsum("qdf,d->qf", 0.5 * (euler.euler_flux(QR) + euler.euler_flux(QL)), -n) + euler.roe_upwind(QR, QL, -n)
    assert np.allclose(fl, -fr, atol=1e-13)


def test_farfield_state_at_freestream():
    """The farfield state of a freestream interior is the freestream, in and out."""
    rho, p, u = 1.0, 1.0 / euler.GAMMA, np.array([0.3, 0.1, 0.0])
    Q = np.array([[rho, *(rho * u), p / (euler.GAMMA - 1) + 0.5 * rho * u @ u]])
    for n in (np.array([1.0, 0, 0]), np.array([-1.0, 0, 0]), np.array([0, 1.0, 0])):
        assert np.allclose(euler.farfield_state(Q, n, rho, p, u), Q, atol=1e-14)


def test_mass_conservation():
    """Interior face fluxes cancel: the sum of every element's mean-mode
    residual equals the flux through the boundary faces."""
    b = euler.EulerBox(3, 3, 2, 1, vel_inf=(0.3, 0.05, 0.02))
    q = b.density_bump(amplitude=0.05, width=0.3, centre=(0.4, 0.5, 0.5))
    R = b.residual(q).reshape(b.nelem, 5, b.nterms)
    U = b.modes(q)
    total = np.zeros(5)
    for fid in range(6):
        E = b._boundary_elems(fid)
        Qm = np.einsum("qm,efm->eqf", b.phif[fid], U[E])
        total += np.einsum("q,pqf->f", b.wf, b._bc_integrand(fid)(Qm))
    assert np.allclose(R[:, :, 0].sum(0), total, atol=1e-14)


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


@pytest.mark.parametrize("bcs", ["farfield", ["farfield", "extrapolate"] * 3])
@pytest.mark.parametrize("P", [1, 2])
def test_jacobian_is_derivative_of_residual(bcs, P):
    """dR/dq against central differences of R along a random direction, with
    the freestream oblique to every face (so that no farfield node sits on the
    inflow/outflow switch, where R is not differentiable)."""
    b = euler.EulerBox(3, 2, 2, P, bcs=bcs, vel_inf=(0.3, 0.1, -0.07))
    q = b.density_bump(amplitude=0.05, width=0.3, centre=(0.4, 0.5, 0.5))
    R, vals = b.residual(q, jacobian=True)
    assert np.allclose(R, b.residual(q), atol=1e-15)
    J = dense(b.pattern, vals)
    v = np.random.default_rng(5).standard_normal(q.size)
    eps = 1e-6
    fd = (b.residual(q + eps * v) - b.residual(q - eps * v)) / (2 * eps)
    assert np.linalg.norm(J @ v - fd) <= 1e-8 * np.linalg.norm(fd)


def test_jacobian_fills_the_box_pattern():
    b = euler.EulerBox(3, 3, 3, 1)
    q = b.density_bump(amplitude=0.05, width=0.3)
    _, vals = b.residual(q, jacobian=True)
    voff, _ = b.pattern.value_offsets()
    nrm = np.array([np.abs(vals[o:o + 1600]).max() for o in voff])
    assert (nrm > 0).all() and vals.size == b.pattern.value_offsets()[1]


def test_pseudo_timestep_at_freestream():
    b = euler.EulerBox(2, 2, 2, 1, extent=((0, 1), (0, 2), (0, 4)))
    q = b.freestream()
    dtau = b.pseudo_timestep(q, np.arange(1.0, 6.0))
    h = b.vol ** (1 / 3)
    lam = 0.3 + 1.0                                   # |u| + c with rho = 1, p = 1/gamma
    assert dtau.shape == (8, 5)
    assert np.allclose(dtau, np.arange(1.0, 6.0)[None, :] * h / lam)


def test_bad_arguments():
    with pytest.raises(ValueError):
        euler.EulerBox(2, 2, 2, 4)
    with pytest.raises(ValueError):
        euler.EulerBox(2, 2, 2, 1, bcs="wall")


def test_add_pseudo_time_matches_dense():
    """euler.add_pseudo_time (the host counterpart of scale_diagonal) adds
    mass / min_f dtau[e, f] to each field's diagonal sub-block of DIAG, nothing
    else (the reference applies minval(elems(ielem)%dtau) to every field)."""
    b = euler.EulerBox(3, 2, 2, 1)
    q = b.density_bump(amplitude=0.05, width=0.3)
    _, vals = b.residual(q, jacobian=True)
    dtau = b.pseudo_timestep(q, [1.0, 2.0, 3.0, 4.0, 5.0])
    got = dense(b.pattern, euler.add_pseudo_time(b, vals, dtau))
    want = dense(b.pattern, vals)
    nt = b.nterms
    for e in range(b.nelem):
        for f in range(5):
            s = (e * 5 + f) * nt
            want[s:s + nt, s:s + nt] += b.mass_block / dtau[e].min()
    assert np.allclose(got, want, rtol=0, atol=1e-15 * np.abs(want).max())


def dense_levels(pat, vals):
    """dense() with time levels: element-major, then time level, field, mode."""
    n = pat.vector_size()
    J = np.zeros((n, n))
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    eo, b = pat.elem_offsets(), pat.bsize()
    for k in range(pat.nblocks):
        r0 = eo[pat.blk_row_elem[k]] + pat.blk_row_time[k] * b[pat.blk_row_elem[k]]
        c0 = eo[pat.blk_col_elem[k]] + pat.blk_col_time[k] * b[pat.blk_col_elem[k]]
        J[r0:r0 + nr[k], c0:c0 + nc[k]] += vals[voff[k]:voff[k] + nr[k] * nc[k]].reshape(nc[k], nr[k]).T
    return J


def test_hb_operator_differentiates_its_harmonics():
    """D (mod_HB_matrices.f90) maps samples of 1, sin w t, cos w t at the time
    levels (type_time_manager.f90) to the samples of their derivatives."""
    w = np.array([1.3, 2.6])
    t = euler.hb_times(w)
    assert t.size == 5 and np.isclose(t[-1], 2 * np.pi / 1.3)
    D = euler.hb_operator(w, t)
    for wk in w:
        assert np.allclose(D @ np.sin(wk * t), wk * np.cos(wk * t), atol=1e-13)
        assert np.allclose(D @ np.cos(wk * t), -wk * np.sin(wk * t), atol=1e-13)
    assert np.allclose(D @ np.ones(5), 0.0, atol=1e-13)


def test_hb_freestream_and_jacobian():
    """Steady farfield: every level at freestream has a zero residual.  With a
    sinusoidal inflow, dR/dq (spatial blocks per level + D(t, t') mass in the
    hb blocks) against central differences of R."""
    hb = euler.EulerHB(3, 2, 2, 1, [1.0], amplitude=0.0, vel_inf=(0.3, 0.1, -0.05))
    assert np.abs(hb.residual(hb.freestream())).max() < 1e-13
    hb = euler.EulerHB(3, 2, 2, 1, [1.0, 2.0], amplitude=0.05, vel_inf=(0.3, 0.1, -0.07))
    assert hb.ntime == 5 and hb.pattern.ntime == 5
    q = hb.density_bump(amplitude=0.05, width=0.3, centre=(0.4, 0.5, 0.5))
    R, vals = hb.residual(q, jacobian=True)
    assert np.allclose(R, hb.residual(q), atol=1e-15)
    J = dense_levels(hb.pattern, vals)
    v = np.random.default_rng(7).standard_normal(q.size)
    eps = 1e-6
    fd = (hb.residual(q + eps * v) - hb.residual(q - eps * v)) / (2 * eps)
    assert np.linalg.norm(J @ v - fd) <= 1e-8 * np.linalg.norm(fd)
    # the pseudo-transient term reaches the DIAG block of every level
    d = hb.pseudo_timestep(q, 10.0)
    added = dense_levels(hb.pattern, hb.add_pseudo_time(vals, d)) - J
    nt, T = hb.nterms, hb.ntime
    want = np.zeros_like(added)
    for e in range(hb.nelem):
        for t in range(T):
            for f in range(5):
                s = ((e * T + t) * 5 + f) * nt
                want[s:s + nt, s:s + nt] = hb.base.mass_block / d[e].min()
    assert np.allclose(added, want, atol=1e-15 * np.abs(want).max())
