"""Host logic of the Newton driver (no GPU calls)."""
import pytest

from chidg_b200.newton import Newton, NewtonOptions


def test_defaults_follow_nonlinear_solver_t():
    """type_nonlinear_solver.f90:21-36, smoothing off as the input namelist
    sets it (mod_io.f90:74-77)."""
    o = NewtonOptions()
    assert (o.cfl0, o.cfl_max, o.cfl_up, o.cfl_down, o.tol, o.rtol, o.nmax, o.ptc, o.search) == \
        (1.0, -1.0, 1.5, 0.1, 1e-10, 1e-10, -1, True, "backtrack")
    assert (o.smooth, o.smoother, o.nsmooth, o.smooth_relax) == (False, "jacobi", 3, 1.0)


def test_refuses_unknown_smoother_and_search():
    Newton(smooth=True, smoother="preconditioner")
    with pytest.raises(ValueError):
        Newton(smooth=True, smoother="gauss-seidel")
    with pytest.raises(ValueError):
        Newton(search="linesearch")


# ---------------------------------------------------------------------------
# the host Newton restatement (oracle/newton_oracle.py) that the GPU driver is
# checked against, itself checked against a dense loop with exact solves
# ---------------------------------------------------------------------------
class _HostSynthetic:
    """R(q) = A0 (q - q*) + c (q - q*)^2 on the host: identity mass matrices and
    dtau = cfl, so the pseudo-transient term adds I / cfl."""

    def __init__(self, pat, seed, c, root_seed):
        import numpy as np

        from chidg_b200 import mesh
        from tests.test_gpu_newton import dense
        self.pat = self.pattern = pat
        self.c = c
        self.values0 = mesh.synth_values(pat, seed=seed)
        self.qstar = 0.3 * mesh.synth_vector(pat.vector_size(), seed=root_seed)
        self.A0 = dense(pat, self.values0)
        voff, _ = pat.value_offsets()
        nr, _ = pat.block_dims()
        eo, b = pat.elem_offsets(), pat.bsize()
        pos, idx = [], []
        for k in np.nonzero((pat.blk_row_elem == pat.blk_col_elem) & (pat.blk_kind == 0))[0]:
            e, n = int(pat.blk_row_elem[k]), int(nr[k])
            pos.append(voff[k] + np.arange(n) * (n + 1))
            idx.append(eo[e] + np.arange(n))
        self.pos, self.idx = np.concatenate(pos), np.concatenate(idx)

    def residual(self, q, jacobian=False):
        d = q - self.qstar
        R = self.A0 @ d + self.c * d * d
        if not jacobian:
            return R
        v = self.values0.copy()
        v[self.pos] += 2.0 * self.c * d[self.idx]
        return R, v

    def pseudo_timestep(self, q, cfl):
        import numpy as np
        return np.full((self.pat.nelem, 1), float(np.mean(cfl)))

    def add_pseudo_time(self, vals, dtau):
        v = vals.copy()
        v[self.pos] += 1.0 / dtau[0, 0]
        return v

    @property
    def mass_block(self):
        import numpy as np
        return np.eye(int(self.pat.elem_nterms[0]))


@pytest.mark.parametrize("ptc,c,cfl0,smooth", [(True, 0.2, 100.0, False), (False, 0.2, 100.0, False),
                                                (True, 2.0, 1.0, False), (True, 0.2, 100.0, True),
                                                (True, 1.0, 5.0, True)])
def test_host_newton_oracle_matches_dense_loop(ptc, c, cfl0, smooth):
    import numpy as np

    from chidg_b200 import mesh
    from oracle import newton_oracle
    from tests.test_gpu_newton import newton_numpy
    pat = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    sysm = _HostSynthetic(pat, seed=121, c=c, root_seed=122)
    opts = dict(tol=1e-9, rtol=1e-12, nmax=40, ptc=ptc, cfl0=cfl0, smooth=smooth, smooth_relax=0.5 if smooth else 1.0)
    res = newton_oracle.newton(sysm, pat, np.zeros(pat.vector_size()), **opts,
                               linear_opts=dict(tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=400))
    qn, hist, alphas = newton_numpy(sysm, np.zeros(pat.vector_size()), NewtonOptions(**opts))
    m = min(len(hist), len(res["residual_norm"]), 4)
    for k in range(m):
        if hist[k] > 1e-6:
            assert abs(res["residual_norm"][k] - hist[k]) <= 1e-6 * hist[k]
    assert res["alphas"][:4] == alphas[:4]
    assert np.linalg.norm(res["q"] - sysm.qstar) <= 1e-6 * np.linalg.norm(sysm.qstar)
