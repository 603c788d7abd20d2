"""The project autotuner (chidg_gpu_autotune via chidg_b200.tuning): it picks
a valid shape for every streamed kernel kind, the solve that follows still
matches the oracle, and a cache file written by one tuning is loaded by the
next without measuring again."""
import json
import time

import numpy as np
import pytest

from chidg_b200 import api, mesh, tuning
from oracle import oracle as O

pytestmark = pytest.mark.gpu

OPTS = dict(tol=0.0, rtol=1e-10, nkrylov=20, inner_fgmres=0, nmax=400)


@pytest.fixture(autouse=True)
def _restore_shapes():
    """The shape table belongs to the process: put it back as it was, so the
    tests that run later see the default shapes."""
    keys = [(k, b, w) for k in tuning.KINDS for b in tuning.CLASSES for w in (8, 4, 2)]
    saved = {key: tuning.get_shape(*key) for key in keys}
    yield
    for key, sh in saved.items():
        tuning.set_shape(*key, sh)


def _system(P=2):
    pat = mesh.box_pattern(6, 5, 4, 5, mesh.nterms_of_order(P))
    return pat, mesh.synth_values(pat, seed=61), mesh.synth_vector(pat.vector_size(), seed=62)


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_autotune_keeps_the_solve_exact(precision, tmp_path):
    pat, vals, b = _system()
    A = api.ChidgMatrix(pat)
    A.upload(vals)
    M = api.create_preconditioner("ilu0")
    M.update(A, precision=precision)
    cache = str(tmp_path / "shapes.json")
    shapes = tuning.autotune(A, M, precision, reps=1, cache=cache)
    assert len(shapes) == 4
    for sh in shapes.values():
        assert sh["warps"] in (4, 8, 16) and 2 <= sh["stages"] <= 8 and sh["stage_bytes"] >= 135 * 2 + 16
    with open(cache) as f:
        assert json.load(f) == shapes
    t0 = time.perf_counter()
    again = tuning.autotune(A, M, precision, reps=1, cache=cache)      # loaded, not measured
    assert again == shapes and time.perf_counter() - t0 < 1.0
    x = api.ChidgVector(A)
    s = api.create_linear_solver("fgmres", **OPTS, **({"precision": precision} if precision != "fp64" else {}))
    s.solve(A, x, api.ChidgVector(A, b), M)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), b, O.default_opts(**OPTS))
    err = np.linalg.norm(x.download() - xo) / np.linalg.norm(xo)
    if precision == "fp64":
        assert s.niter == ro["niter"] and err < 1e-10
    else:
        assert s.residual_norm <= 1.0001e-10 * s.r0norm_initial and err < 1e-8


def test_shape_set_refuses_bad_shapes():
    from chidg_b200 import _lib
    L = _lib.lib()
    assert L.chidg_gpu_stream_shape_set(0, 135, 8, 5, 2, 24576) == _lib.EINVAL      # warps
    assert L.chidg_gpu_stream_shape_set(0, 135, 8, 8, 1, 24576) == _lib.EINVAL      # stages
    assert L.chidg_gpu_stream_shape_set(0, 135, 3, 8, 2, 24576) == _lib.EINVAL      # value width
    assert L.chidg_gpu_stream_shape_set(9, 135, 8, 8, 2, 24576) == _lib.EINVAL      # kind
