"""The oracle's host threads change no bit of its results: matvec, ILU0 and
RAS+ILU0 factors and sweeps, A^T products and factors, and the FGMRES history,
for one thread against several (CPU only)."""
import numpy as np
import pytest

from chidg_b200 import mesh
from oracle import oracle as O


def _system(subdomains=(1, 1, 1)):
    pat = mesh.box_pattern(4, 4, 3, 5, mesh.nterms_of_order(1), subdomains=subdomains)
    return pat, mesh.synth_values(pat, seed=31), mesh.synth_vector(pat.vector_size(), seed=32)


def _run(threads, kind, transposed=False, subdomains=(1, 1, 1)):
    pat, vals, b = _system(subdomains)
    O.set_threads(threads)
    try:
        A = O.OracleMatrix(pat)
        A.set_values(vals)
        A.set_transposed(transposed)
        M = O.OraclePrecon(A, kind)
        M.update()
        x, res = O.fgmres(A, O.OraclePrecon(A, kind), b, O.default_opts(tol=0.0, rtol=1e-10, nkrylov=20,
                                                                         inner_fgmres=0, nmax=400))
        return [A.mv(b), M.LD(), M.apply(b), x, res["hist"]]
    finally:
        O.set_threads(1)


@pytest.mark.parametrize("kind,transposed,subdomains", [("ilu0", False, (1, 1, 1)), ("ilu0", True, (1, 1, 1)),
                                                        ("jacobi", False, (1, 1, 1)),
                                                        ("rasilu0", False, (2, 2, 1))])
def test_threads_are_bitwise_neutral(kind, transposed, subdomains):
    one = _run(1, kind, transposed, subdomains)
    many = _run(4, kind, transposed, subdomains)
    for a, b in zip(one, many):
        assert np.array_equal(a, b)


def test_thread_count_is_checked():
    with pytest.raises(ValueError):
        O.set_threads(0)
    O.set_threads(2)
    assert O.get_threads() == 2
    O.set_threads(1)
