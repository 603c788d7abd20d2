"""The oracle replays the reference's own known-answer tests (parity pin)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import kat_util

CASES = kat_util.load_cases()


@pytest.mark.parametrize("name", ["ilu0", "ilu0_hb"])
def test_ilu0_kat(name):
    case = CASES[name]
    pat, vals, b = kat_util.build(case)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    M = O.OraclePrecon(A, "ilu0")
    M.update()
    LD = M.LD()
    n_ld = 0
    for kind, idx, expect in case["asserts"]:
        if kind == "LD":
            # pFUnit @assertEqual without tolerance: exact
            assert LD[kat_util.ld_index(pat, *idx)] == pytest.approx(expect, rel=1e-15, abs=0), (idx, expect)
            n_ld += 1
    assert n_ld >= 5
    z = M.apply(b)
    eo = pat.elem_offsets()
    n_z = 0
    for kind, idx, expect in case["asserts"]:
        if kind == "z":
            e, i = idx
            assert abs(z[eo[e - 1] + i - 1] - expect) <= case["tol"]
            n_z += 1
    assert n_z >= 3


@pytest.mark.parametrize("name", ["fgmres", "fgmres_ref"])
def test_fgmres_kat(name):
    case = CASES[name]
    pat, vals, b = kat_util.build(case)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    M = O.OraclePrecon(A, "identity")
    # reference defaults (inner_fgmres on) with linear_solver%tol = 1e-13
    x, res = O.fgmres(A, M, b, O.default_opts(tol=case["solver_tol"], nmax=1000))
    eo = pat.elem_offsets()
    for kind, (e, i), expect in case["asserts"]:
        assert kind == "x"
        assert abs(x[eo[e - 1] + i - 1] - expect) <= case["tol"]
    assert res["residual_norm"] < 1e-12


@pytest.mark.parametrize("name", ["mv", "mtv", "mtv_2"])
def test_operator_kat(name):
    """test_chidg_matrix_operator_mv.pf / _mtv.pf: chidg_mv and the
    transposed product (chidg_matrix_t%transposed) on LOCAL and CHIMERA blocks."""
    case = CASES[name]
    pat, vals, x = kat_util.build_operator(case)
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    if case["mode"] == "mtv":
        A.set_transposed(True)
    y = A.mv(x)
    eo = pat.elem_offsets()
    for e, expect in case["asserts"]:
        assert np.all(np.abs(y[eo[e]:eo[e + 1]] - expect) <= case["tol"]), (e, expect, y[eo[e]:eo[e + 1]])
    assert len(case["asserts"]) >= 2


def test_inv_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (1, 2, 5, 40, 135):
        a = rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n)
        assert np.allclose(O.inv(a), np.linalg.inv(a), rtol=1e-10, atol=1e-12)


def test_inv_singular():
    with pytest.raises(ArithmeticError):
        O.inv(np.zeros((3, 3)))
