"""Host-side pieces of bench.py (no GPU): the seeded Euler box of the
configurations and the host-assembled Newton system that the CPU baseline and
the reference arm solve with the oracle."""
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


def test_cpu_sample_system_is_solved_by_the_oracle():
    pat, vals, b = bench.cpu_sample_system(n=3)
    assert vals.size == pat.value_offsets()[1] and b.size == pat.vector_size()
    A = O.OracleMatrix(pat)
    A.set_values(vals)
    dt, niter = bench.cpu_sample_solve((pat, vals, b), A)
    assert dt > 0.0 and 0 < niter < bench.SOLVER["nmax"]
    opts = {k: v for k, v in bench.SOLVER.items() if k != "orthogonalization"}
    x, res = O.fgmres(A, O.OraclePrecon(A, "ilu0"), b, O.default_opts(**opts))
    assert np.linalg.norm(A.mv(x) - b) <= 1e-8 * np.linalg.norm(b) * 1.0001
