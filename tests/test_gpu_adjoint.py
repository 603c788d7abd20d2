"""GPU parity of the transposed operators (chidg_matrix_t%transposed, the
adjoint path): A^T x, ILU0 / Jacobi of A^T, FGMRES on A^T x = b, against the
oracle's restatement of the reference's transposed branches and the
reference's own mtv known-answer tests.

Tolerances as in the other FP64 parity tests: products 1e-13 relative, sweeps
1e-11, factor blocks 1e-10 relative to the block norm, FGMRES same iteration
count, history 1e-8 and solution 1e-10 relative.
"""
import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh
from oracle import oracle as O
from tests import kat_util

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def setup(shape, P, nt=1, sub=(1, 1, 1), seed=1, transposed=True):
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt, subdomains=sub)
    vals = mesh.synth_values(pat, seed=seed)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(pat)
    Ag.upload(vals)
    if transposed:
        Ao.set_transposed(True)
        Ag.transposed = True
    return pat, vals, Ao, Ag


@pytest.mark.parametrize("shape,P,nt", [((3, 3, 2), 1, 1), ((2, 2, 2), 2, 1), ((2, 2, 2), 1, 3), ((2, 2, 1), 3, 1)])
def test_transposed_matvec_matches_oracle(shape, P, nt):
    """transposed_matrix_vector_product, harmonic-balance blocks included."""
    pat, vals, Ao, Ag = setup(shape, P, nt, seed=41)
    assert Ag.transposed
    x = mesh.synth_vector(Ao.n, seed=42)
    y = api.chidg_mv(Ag, api.ChidgVector(Ag, x)).download()
    assert relerr(y, Ao.mv(x)) < 1e-13


@pytest.mark.parametrize("order", ["reference", "by_column"])
@pytest.mark.parametrize("name", ["mv", "mtv", "mtv_2"])
def test_operator_kat(name, order):
    """The reference's test_chidg_matrix_operator_mv / _mtv known answers,
    LOCAL and CHIMERA blocks, through the C ABI; with the blocks listed in the
    reference's order (streamed matvec) and by column (rows not contiguous in
    the packed values: the one-CTA-per-row matvec)."""
    case = kat_util.load_cases()[name]
    pat, vals, x = kat_util.build_operator(case, order)
    A = api.ChidgMatrix(pat)
    A.upload(vals)
    if case["mode"] == "mtv":
        A.transposed = True
    y = api.chidg_mv(A, api.ChidgVector(A, x)).download()
    eo = pat.elem_offsets()
    for e, expect in case["asserts"]:
        assert np.all(np.abs(y[eo[e]:eo[e + 1]] - expect) <= case["tol"]), (e, expect)


@pytest.mark.parametrize("kind,nt,schedule", [("ilu0", 1, "stream"), ("ilu0", 1, "tasks"), ("ilu0", 2, "stream"),
                                              ("jacobi", 1, "stream")])
def test_transposed_precon_matches_oracle(kind, nt, schedule):
    """precon_ILU0.f90:148-207,378-383 and precon_jacobi.f90:121-125."""
    pat, vals, Ao, Ag = setup((3, 3, 2), 1, nt, seed=43)
    Mo = O.OraclePrecon(Ao, kind)
    Mo.update()
    Mg = api.create_preconditioner(kind, schedule=schedule)
    Mg.update(Ag)
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    LDg, LDo = Mg.LD(), Mo.LD()
    for k in range(pat.nblocks):
        sl = slice(voff[k], voff[k] + nr[k] * nc[k])
        assert np.linalg.norm(LDg[sl] - LDo[sl]) <= 1e-10 * max(np.linalg.norm(LDo[sl]), 1e-300), k
    v = mesh.synth_vector(Ao.n, seed=44)
    assert relerr(Mg.apply(Ag, api.ChidgVector(Ag, v)).download(), Mo.apply(v)) < 1e-11


def test_transposed_fgmres_matches_oracle():
    pat, vals, Ao, Ag = setup((4, 3, 2), 1, seed=45)
    b = mesh.synth_vector(Ao.n, seed=46)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=20, inner_fgmres=0, nmax=400)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), b, O.default_opts(**opts))
    solver = api.create_linear_solver("fgmres", **opts)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("ilu0"))
    assert solver.niter == ro["niter"]
    assert relerr(solver.hist, ro["hist"]) < 1e-8
    assert relerr(xg.download(), xo) < 1e-10
    # x solves the adjoint system: A^T x = b
    assert relerr(Ao.mv(xg.download()), b) < 2e-8


@pytest.mark.parametrize("precision", ["mixed_fp32", "mixed_bf16", "mixed_precon_fp32"])
def test_transposed_mixed_precision_reaches_fp64_accuracy(precision):
    pat, vals, Ao, Ag = setup((4, 4, 4), 1, seed=47)
    b = mesh.synth_vector(Ao.n, seed=48)
    xo, _ = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), b,
                     O.default_opts(tol=0.0, rtol=1e-12, nkrylov=40, inner_fgmres=0, nmax=400))
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=50,
                                      precision=precision, mixed_inner_nkrylov=20, mixed_inner_rtol=1e-2,
                                      mixed_inner_nmax=40)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("ilu0"))
    assert solver.residual_norm <= 1.5e-8 * solver.r0norm_initial
    assert relerr(xg.download(), xo) < 1e-6


def test_transposed_batched_matches_single_oracle_solves():
    systems = [((3, 3, 2), 1, 51), ((2, 2, 2), 2, 52), ((3, 2, 2), 1, 53)]
    pats = [mesh.box_pattern(*s, 5, mesh.nterms_of_order(P)) for s, P, _ in systems]
    vals = [mesh.synth_values(p, seed=sd) for p, (_, _, sd) in zip(pats, systems)]
    rhs = [mesh.synth_vector(p.vector_size(), seed=sd + 100) for p, (_, _, sd) in zip(pats, systems)]
    union, sys_elem = mesh.concat_patterns(pats)
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    A.transposed = True
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=300)
    res = api.create_linear_solver("fgmres", **opts).solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
    xg = x.download()
    off = 0
    for s, (pat, v, r) in enumerate(zip(pats, vals, rhs)):
        Ao = O.OracleMatrix(pat)
        Ao.set_values(v)
        Ao.set_transposed(True)
        xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), r, O.default_opts(**opts))
        n = pat.vector_size()
        assert res[s]["niter"] == ro["niter"]
        assert relerr(xg[off:off + n], xo) < 1e-10
        off += n


def test_rasilu0_refuses_transposed_matrix():
    """precon_RASILU0.f90:254: transpose not implemented for native containers."""
    pat, vals, Ao, Ag = setup((4, 2, 2), 1, sub=(2, 1, 1), seed=55)
    M = api.create_preconditioner("rasilu0")
    with pytest.raises(_lib.ChidgGpuError) as ei:
        M.update(Ag)
    assert ei.value.code == _lib.EINVAL


def test_flag_toggle_and_value_refresh():
    """A preconditioner made before the flag is set rebuilds its programme at
    its next update; new values reach A^T; clearing the flag restores A."""
    pat, vals, Ao, Ag = setup((3, 2, 2), 1, seed=57, transposed=False)
    M = api.create_preconditioner("ilu0")
    M.update(Ag)
    x = mesh.synth_vector(Ao.n, seed=58)
    xv = api.ChidgVector(Ag, x)
    forward = api.chidg_mv(Ag, xv).download()
    assert relerr(forward, Ao.mv(x)) < 1e-13
    Ag.transposed = True
    Ao.set_transposed(True)
    assert relerr(api.chidg_mv(Ag, xv).download(), Ao.mv(x)) < 1e-13
    M.update(Ag)
    Mo = O.OraclePrecon(Ao, "ilu0")
    Mo.update()
    assert relerr(M.apply(Ag, xv).download(), Mo.apply(x)) < 1e-11
    vals2 = mesh.synth_values(pat, seed=59)
    Ag.upload(vals2)
    Ao.set_values(vals2)
    assert relerr(api.chidg_mv(Ag, xv).download(), Ao.mv(x)) < 1e-13
    Ag.transposed = False
    Ao.set_transposed(False)
    assert relerr(api.chidg_mv(Ag, xv).download(), Ao.mv(x)) < 1e-13
    M.update(Ag)
    Mo = O.OraclePrecon(Ao, "ilu0")
    Mo.update()
    assert relerr(M.apply(Ag, xv).download(), Mo.apply(x)) < 1e-11


def test_mixed_precision_with_identity_preconditioner():
    """The FP32 copy of A read by the inner solves exists without a factorisation."""
    pat, vals, Ao, Ag = setup((2, 2, 2), 1, seed=61, transposed=False)
    b = mesh.synth_vector(Ao.n, seed=62)
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=60,
                                      precision="mixed_fp32", mixed_inner_nkrylov=30, mixed_inner_rtol=1e-2,
                                      mixed_inner_nmax=60)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("identity"))
    assert solver.residual_norm <= 1.5e-8 * solver.r0norm_initial
