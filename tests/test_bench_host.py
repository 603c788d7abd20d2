"""Host-side pieces of bench.py (no GPU): the seeded Euler box of the
configurations and the host-assembled Newton system that the reference arm
solves with the oracle."""
import numpy as np

import bench
from oracle import oracle as O


def test_euler_box_seeding():
    box, q0, centre = bench.euler_box(3, seed=5, order=1, mach=0.4)
    assert box.shape == (3, 3, 3) and box.order == 1
    assert np.all((centre >= 0.3) & (centre <= 0.7))
    assert box.vel_inf == (0.4, 0.0, 0.0)
    _, _, centre2 = bench.euler_box(3, seed=5, order=1)
    assert np.array_equal(centre, centre2)                  # the centre depends on the seed only


def test_host_newton_system_is_solved_by_the_oracle():
    pat, vals, b = bench.host_newton_system(n=3)
    assert vals.size == pat.value_offsets()[1] and b.size == pat.vector_size()
    A = bench.oracle_matrix(pat, vals)
    dt, x, res = bench.oracle_solve(A, b)
    assert dt > 0.0 and 0 < res["niter"] < bench.SOLVER["nmax"]
    assert np.linalg.norm(A.mv(x) - b) <= 1e-8 * np.linalg.norm(b) * 1.0001


def test_oracle_threads_give_the_one_thread_solution():
    """The reference arm runs the oracle on every host thread; its solution is
    bitwise the one-thread solution."""
    pat, vals, b = bench.host_newton_system(n=4, order=1)
    out = []
    for threads in (1, 3):
        O.set_threads(threads)
        A = bench.oracle_matrix(pat, vals)
        out.append(bench.oracle_solve(A, b)[1:])
    O.set_threads(1)
    (x1, r1), (x3, r3) = out
    assert np.array_equal(x1, x3) and np.array_equal(r1["hist"], r3["hist"])
