"""Host logic of the Newton driver (no GPU calls)."""
import pytest

from chidg_b200.newton import Newton, NewtonOptions


def test_defaults_follow_nonlinear_solver_t():
    """type_nonlinear_solver.f90:21-36 (residual smoothing is not restated)."""
    o = NewtonOptions()
    assert (o.cfl0, o.cfl_max, o.cfl_up, o.cfl_down, o.tol, o.rtol, o.nmax, o.ptc, o.search) == \
        (1.0, -1.0, 1.5, 0.1, 1e-10, 1e-10, -1, True, "backtrack")


def test_refuses_smoothing_and_unknown_search():
    with pytest.raises(NotImplementedError):
        Newton(smooth=True)
    with pytest.raises(ValueError):
        Newton(search="linesearch")
