"""Oracle vs independent dense numpy restatements on small seeded systems."""
import numpy as np
import pytest

from chidg_b200 import mesh
from oracle import oracle as O


def dense(pat, vals):
    """Assemble the full matrix from the packed blocks."""
    n = pat.vector_size()
    D = np.zeros((n, n))
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    eo = pat.elem_offsets()
    b = pat.bsize()
    for k in range(pat.nblocks):
        r0 = eo[pat.blk_row_elem[k]] + pat.blk_row_time[k] * b[pat.blk_row_elem[k]]
        c0 = eo[pat.blk_col_elem[k]] + pat.blk_col_time[k] * b[pat.blk_col_elem[k]]
        blk = vals[voff[k]:voff[k] + nr[k] * nc[k]].reshape(nc[k], nr[k]).T
        D[r0:r0 + nr[k], c0:c0 + nc[k]] += blk
    return D


def block_ilu0_dense(pat, vals):
    """Block ILU(0) on the LOCAL-block pattern in natural order, dense numpy."""
    D = dense(pat, vals)
    b = int(pat.bsize()[0])
    nt = pat.ntime
    nrow = pat.nelem * nt
    blk = lambda r, c: D[r * b:(r + 1) * b, c * b:(c + 1) * b]
    local = set()
    for k in range(pat.nblocks):
        if pat.blk_kind[k] == 0:
            local.add((pat.blk_row_elem[k] * nt + pat.blk_row_time[k], pat.blk_col_elem[k] * nt + pat.blk_col_time[k]))
    Dinv, L = {}, {}
    for r in range(nrow):
        Dr = blk(r, r).copy()
        for c in sorted(c for (rr, c) in local if rr == r and c < r):
            L[(r, c)] = blk(r, c) @ Dinv[c]
            Dr -= L[(r, c)] @ blk(c, r)
        Dinv[r] = np.linalg.inv(Dr)
    return Dinv, L, local, blk


@pytest.mark.parametrize("shape,P,nt", [((3, 2, 2), 1, 1), ((2, 2, 2), 0, 3), ((4, 1, 1), 1, 1)])
def test_mv_matches_dense(shape, P, nt):
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt)
    vals = mesh.synth_values(pat, seed=3)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    x = mesh.synth_vector(A.n, seed=4)
    assert np.allclose(A.mv(x), dense(pat, vals) @ x, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("shape,P,nt", [((3, 2, 2), 1, 1), ((2, 2, 2), 0, 2)])
def test_ilu0_matches_dense(shape, P, nt):
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt)
    vals = mesh.synth_values(pat, seed=5)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    M = O.OraclePrecon(A, "ilu0")
    M.update()
    Dinv, L, local, blk = block_ilu0_dense(pat, vals)
    v = mesh.synth_vector(A.n, seed=6)
    # apply: forward with L, backward with A's upper blocks, then Dinv
    b = int(pat.bsize()[0])
    nrow = pat.nelem * pat.ntime
    z = v.copy().reshape(nrow, b)
    for r in range(nrow):
        for c in sorted(c for (rr, c) in local if rr == r and c < r):
            z[r] -= L[(r, c)] @ z[c]
    for r in reversed(range(nrow)):
        for c in sorted(c for (rr, c) in local if rr == r and c > r):
            z[r] -= blk(r, c) @ z[c]
        z[r] = Dinv[r] @ z[r]
    assert np.allclose(M.apply(v), z.ravel(), rtol=1e-11, atol=1e-12)


def test_fgmres_matches_dense_solve():
    pat = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    vals = mesh.synth_values(pat, seed=7)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    b = mesh.synth_vector(A.n, seed=8)
    x, res = O.fgmres(A, O.OraclePrecon(A, "ilu0"), b,
                      O.default_opts(tol=0.0, rtol=1e-12, nkrylov=30, inner_fgmres=0, nmax=500))
    xd = np.linalg.solve(dense(pat, vals), b)
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
    assert res["residual_norm"] <= 1e-11 * np.linalg.norm(b)
    # history is monotone non-increasing within a cycle (GMRES minimal residual)
    h = res["hist"]
    assert np.all(np.diff(h[:min(len(h), 30)]) <= 1e-12 * h[0])


def test_rasilu0_single_subdomain_equals_ilu0():
    pat = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    vals = mesh.synth_values(pat, seed=9)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    v = mesh.synth_vector(A.n, seed=10)
    M1 = O.OraclePrecon(A, "ilu0")
    M1.update()
    M2 = O.OraclePrecon(A, "rasilu0")
    M2.update()
    assert np.allclose(M1.apply(v), M2.apply(v), rtol=1e-14, atol=1e-14)


def test_rasilu0_block_jacobi_limit():
    """With no off-subdomain coupling the RAS solve is the per-subdomain ILU0."""
    pat = mesh.box_pattern(4, 2, 2, 5, mesh.nterms_of_order(0), subdomains=(2, 1, 1))
    vals = mesh.synth_values(pat, seed=11)
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    proc = pat.elem_proc
    cut = vals.copy()
    for k in range(pat.nblocks):
        if proc[pat.blk_row_elem[k]] != proc[pat.blk_col_elem[k]]:
            cut[voff[k]:voff[k] + nr[k] * nc[k]] = 0.0
    A = O.OracleMatrix(pat)
    A.set_values(cut)
    M = O.OraclePrecon(A, "rasilu0")
    M.update()
    M1 = O.OraclePrecon(A, "ilu0")
    M1.update()
    v = mesh.synth_vector(A.n, seed=12)
    # elements are ordered globally, subdomains split along xi, so the
    # global natural-order ILU0 of the decoupled matrix is the same operator
    assert np.allclose(M.apply(v), M1.apply(v), rtol=1e-12, atol=1e-13)


def test_rasilu0_reduces_residual():
    pat = mesh.box_pattern(4, 4, 2, 5, mesh.nterms_of_order(1), subdomains=(2, 2, 1))
    vals = mesh.synth_values(pat, seed=13)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    b = mesh.synth_vector(A.n, seed=14)
    x, res = O.fgmres(A, O.OraclePrecon(A, "rasilu0"), b,
                      O.default_opts(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=300))
    assert res["residual_norm"] <= 2e-8 * res["r0norm_initial"]
    _, res1 = O.fgmres(A, O.OraclePrecon(A, "jacobi"), b,
                       O.default_opts(tol=0.0, rtol=1e-8, nkrylov=30, inner_fgmres=0, nmax=300))
    assert res["niter"] <= res1["niter"]


def transposed_values(pat, vals):
    """Values of A^T on A's own pattern: block (r, c) holds the transpose of
    block (c, r) (box patterns are structurally symmetric, HB blocks included)."""
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    where = {(int(pat.blk_row_elem[k]), int(pat.blk_row_time[k]), int(pat.blk_col_elem[k]),
              int(pat.blk_col_time[k]), int(pat.blk_kind[k])): k for k in range(pat.nblocks)}
    out = np.empty_like(vals)
    for (re_, rt, ce, ct, kd), k in where.items():
        kt = where[(ce, ct, re_, rt, kd)]
        src = vals[voff[kt]:voff[kt] + nr[kt] * nc[kt]].reshape(nc[kt], nr[kt]).T   # block kt, (nr x nc)
        out[voff[k]:voff[k] + nr[k] * nc[k]] = src.T.ravel(order="F")
    return out


@pytest.mark.parametrize("shape,P,nt", [((3, 2, 2), 1, 1), ((2, 2, 2), 0, 3)])
def test_mtv_matches_dense(shape, P, nt):
    """transposed_matrix_vector_product (operator_chidg_mv.f90:692-1049), HB term included."""
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt)
    vals = mesh.synth_values(pat, seed=31)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    A.set_transposed(True)
    x = mesh.synth_vector(A.n, seed=32)
    assert np.allclose(A.mv(x), dense(pat, vals).T @ x, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("kind,nt", [("ilu0", 1), ("ilu0", 2), ("jacobi", 1)])
def test_transposed_factors_are_those_of_the_transpose(kind, nt):
    """precon_ILU0.f90:148-207 / precon_jacobi.f90:121-125: the transposed
    branch factors A^T, so it matches the plain branch run on A^T's values."""
    pat = mesh.box_pattern(3, 2, 2, 5, mesh.nterms_of_order(1), ntime=nt)
    vals = mesh.synth_values(pat, seed=33)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    A.set_transposed(True)
    M = O.OraclePrecon(A, kind)
    M.update()
    B = O.OracleMatrix(pat)
    B.set_values(transposed_values(pat, vals))
    MB = O.OraclePrecon(B, kind)
    MB.update()
    assert np.allclose(M.LD(), MB.LD(), rtol=1e-12, atol=1e-13)
    v = mesh.synth_vector(A.n, seed=34)
    assert np.allclose(M.apply(v), MB.apply(v), rtol=1e-12, atol=1e-13)


def test_transposed_fgmres_solves_the_adjoint_system():
    pat = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    vals = mesh.synth_values(pat, seed=35)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    A.set_transposed(True)
    b = mesh.synth_vector(A.n, seed=36)
    x, res = O.fgmres(A, O.OraclePrecon(A, "ilu0"), b,
                      O.default_opts(tol=0.0, rtol=1e-12, nkrylov=30, inner_fgmres=0, nmax=500))
    xd = np.linalg.solve(dense(pat, vals).T, b)
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


def test_rasilu0_refuses_transposed_matrix():
    """precon_RASILU0.f90:254: transpose not implemented for native containers."""
    pat = mesh.box_pattern(4, 2, 2, 5, mesh.nterms_of_order(0), subdomains=(2, 1, 1))
    A = O.OracleMatrix(pat)
    A.set_values(mesh.synth_values(pat, seed=37))
    A.set_transposed(True)
    M = O.OraclePrecon(A, "rasilu0")
    with pytest.raises(ArithmeticError):
        M.update()


@pytest.mark.parametrize("v,F,E", [
    (1.0, "1.00000000000000", None), (-0.5, "-0.50000000000000", None),
    (123456789.5, "123456789.50000000000000", None), (-123456789.5, "*" * 24, None),
    (0.05, None, "0.50000000000000E-01"), (-0.05, None, "-0.50000000000000E-01"),
    (0.1, None, "0.10000000000000E+00"), (0.0, None, "0.00000000000000E+00"),
    (1e9, None, "0.10000000000000E+10"), (1e-120, None, "0.10000000000000-119"),
    (2.5e200, None, "0.25000000000000+201")])
def test_fortran_edit_descriptors(v, F, E):
    """F24.14 / E24.14 as the Fortran standard defines them (the forms
    messenger%add_to_line writes); leading zero shown, as gfortran does."""
    if F is not None:
        assert O.fortran_F(v).strip() == F
    if E is not None:
        assert O.fortran_E(v).strip() == E


def test_to_file_line_layout():
    """One entry: leading blank, four 25-column centred fields, ',' between."""
    pat = mesh.box_pattern(1, 1, 1, 1, 1)
    line = O.to_file_text(pat, np.array([0.25]))
    assert line == " " + ",".join(["            1            "] * 2 + ["            1            ",
                                                                      "     0.25000000000000    "]) + "\n"


@pytest.mark.parametrize("shape,P,nt", [((2, 2, 1), 1, 3), ((2, 1, 1), 0, 5), ((3, 2, 1), 1, 1)])
def test_hb_precon_matches_dense(shape, P, nt):
    """precon_HB.f90:169-310: per element the inverse of its time-coupled
    block (DIAG blocks and hb_blks), applied to the element's segment."""
    pat = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P), ntime=nt)
    vals = mesh.synth_values(pat, seed=81)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    M = O.OraclePrecon(A, "hb")
    M.update()
    D = dense(pat, vals)
    eo = pat.elem_offsets()
    v = mesh.synth_vector(A.n, seed=82)
    z = np.empty_like(v)
    for e in range(pat.nelem):
        s = slice(eo[e], eo[e + 1])
        z[s] = np.linalg.solve(D[s, s], v[s])      # element block: DIAG + HB blocks only (LOCAL neighbours are off it)
    assert np.allclose(M.apply(v), z, rtol=1e-11, atol=1e-12)


def test_hb_precon_reduces_hb_residual():
    """On a pattern with HB coupling, FGMRES with precon_HB converges."""
    pat = mesh.box_pattern(2, 2, 2, 5, mesh.nterms_of_order(1), ntime=3)
    A = O.OracleMatrix(pat)
    A.set_values(mesh.synth_values(pat, seed=83))
    b = mesh.synth_vector(A.n, seed=84)
    x, res = O.fgmres(A, O.OraclePrecon(A, "hb"), b, O.default_opts(tol=0.0, rtol=1e-10, nkrylov=40, inner_fgmres=0,
                                                                     nmax=400))
    assert res["residual_norm"] <= 1e-9 * res["r0norm_initial"]


def test_ragged_orders_match_dense():
    """Elements of orders 0, 1 and 2 in one matrix (non-square coupling
    blocks): matvec, block ILU0 (dense restatement on element slices) and FGMRES."""
    base = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    pat = mesh.with_element_orders(base, [(e * 7) % 3 for e in range(base.nelem)])
    vals = mesh.synth_values(pat, seed=85)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    D = dense(pat, vals)
    x = mesh.synth_vector(A.n, seed=86)
    assert np.allclose(A.mv(x), D @ x, rtol=1e-13, atol=1e-13)
    eo = pat.elem_offsets()
    sl = [slice(eo[e], eo[e + 1]) for e in range(pat.nelem)]
    local = {(int(pat.blk_row_elem[k]), int(pat.blk_col_elem[k])) for k in range(pat.nblocks) if pat.blk_kind[k] == 0}
    Dinv, L = {}, {}
    for r in range(pat.nelem):
        Dr = D[sl[r], sl[r]].copy()
        for c in sorted(c for (rr, c) in local if rr == r and c < r):
            L[(r, c)] = D[sl[r], sl[c]] @ Dinv[c]
            Dr -= L[(r, c)] @ D[sl[c], sl[r]]
        Dinv[r] = np.linalg.inv(Dr)
    z = mesh.synth_vector(A.n, seed=87)
    v = z.copy()
    for r in range(pat.nelem):
        for c in sorted(c for (rr, c) in local if rr == r and c < r):
            z[sl[r]] -= L[(r, c)] @ z[sl[c]]
    for r in reversed(range(pat.nelem)):
        for c in sorted(c for (rr, c) in local if rr == r and c > r):
            z[sl[r]] -= D[sl[r], sl[c]] @ z[sl[c]]
        z[sl[r]] = Dinv[r] @ z[sl[r]]
    M = O.OraclePrecon(A, "ilu0")
    M.update()
    assert np.allclose(M.apply(v), z, rtol=1e-11, atol=1e-12)
