"""GPU parity of precon_HB (precon_HB.f90:169-310): per element the inverse of
its block over all time levels (DIAG blocks and hb_blks), against the oracle.

Tolerances: apply 1e-10 relative (inverses of up to 280 x 280 element
blocks); FGMRES with the same iteration count and the solution within 1e-10.
"""
import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def setup(shape, P, nt, seed):
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt)
    vals = mesh.synth_values(pat, seed=seed)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(pat)
    Ag.upload(vals)
    return pat, vals, Ao, Ag


@pytest.mark.parametrize("shape,P,nt,schedule", [((2, 1, 1), 0, 5, "stream"), ((3, 2, 1), 1, 1, "stream"),
                                                 ((2, 2, 1), 1, 3, "stream"), ((2, 2, 1), 1, 3, "tasks"),
                                                 ((2, 2, 2), 1, 7, "stream")])
def test_hb_precon_matches_oracle(shape, P, nt, schedule):
    """Element blocks of 25, 40, 120 and 280 rows (small, tensor-core and
    global inverse kernels)."""
    pat, vals, Ao, Ag = setup(shape, P, nt, seed=91)
    Mo = O.OraclePrecon(Ao, "hb")
    Mo.update()
    Mg = api.create_preconditioner("hb", schedule=schedule)
    Mg.update(Ag)
    v = mesh.synth_vector(Ao.n, seed=92)
    assert relerr(Mg.apply(Ag, api.ChidgVector(Ag, v)).download(), Mo.apply(v)) < 1e-10


def test_hb_fgmres_matches_oracle():
    pat, vals, Ao, Ag = setup((3, 2, 2), 1, 3, seed=93)
    b = mesh.synth_vector(Ao.n, seed=94)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=20, inner_fgmres=0, nmax=400)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "hb"), b, O.default_opts(**opts))
    solver = api.create_linear_solver("fgmres", **opts)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("hb"))
    assert solver.niter == ro["niter"]
    assert relerr(solver.hist, ro["hist"]) < 1e-8
    assert relerr(xg.download(), xo) < 1e-10


@pytest.mark.parametrize("precision", ["mixed_fp32", "mixed_precon_fp32"])
def test_hb_mixed_precision_reaches_fp64_accuracy(precision):
    pat, vals, Ao, Ag = setup((3, 3, 2), 1, 3, seed=95)
    b = mesh.synth_vector(Ao.n, seed=96)
    xo, _ = O.fgmres(Ao, O.OraclePrecon(Ao, "hb"), b,
                     O.default_opts(tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=600))
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=60,
                                      precision=precision, mixed_inner_nkrylov=30, mixed_inner_rtol=1e-2,
                                      mixed_inner_nmax=60)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("hb"))
    assert solver.residual_norm <= 1.5e-8 * solver.r0norm_initial
    assert relerr(xg.download(), xo) < 1e-6


def test_hb_singular_element_reports_element():
    pat, vals, Ao, Ag = setup((2, 2, 1), 1, 3, seed=97)
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    bad = vals.copy()
    for k in range(pat.nblocks):        # element 2's whole time-coupled block
        if pat.blk_row_elem[k] == 2 and pat.blk_col_elem[k] == 2:
            bad[voff[k]:voff[k] + nr[k] * nc[k]] = 0.0
    Ag.upload(bad)
    M = api.create_preconditioner("hb")
    with pytest.raises(_lib.ChidgGpuError) as ei:
        M.update(Ag)
    assert ei.value.code == _lib.ESINGULAR and ei.value.element == 2


def test_hb_uses_own_blocks_of_a_transposed_matrix_and_refuses_LD():
    """precon_HB does not consult A%transposed; its factors are not LOCAL-block shaped."""
    pat, vals, Ao, Ag = setup((2, 2, 1), 1, 3, seed=98)
    Ag.transposed = True
    Ao.set_transposed(True)
    Mo = O.OraclePrecon(Ao, "hb")
    Mo.update()
    Mg = api.create_preconditioner("hb")
    Mg.update(Ag)
    v = mesh.synth_vector(Ao.n, seed=99)
    assert relerr(Mg.apply(Ag, api.ChidgVector(Ag, v)).download(), Mo.apply(v)) < 1e-10
    with pytest.raises(_lib.ChidgGpuError) as ei:
        Mg.LD()
    assert ei.value.code == _lib.EINVAL
