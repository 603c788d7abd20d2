"""The matvec rows run inside the streamed backward sweep (the fused pass that
FGMRES takes for z = M v followed by w = A z) give bitwise the results of the
separate launches: the same chunks and per-thread order in every product.
Checked on whole FGMRES solves against a process that runs the separate
launches (CHIDG_FUSED_MV=0), for FP64, FP32 preconditioner blocks and the FP32
and BF16 inner solves, with ILU0 and Jacobi, on one and three time levels."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [("ilu0", "fp64", 1, 2), ("ilu0", "fp64", 3, 1), ("jacobi", "fp64", 1, 1), ("ilu0", "mixed_precon_fp32", 1, 2),
         ("ilu0", "mixed_fp32", 1, 2), ("ilu0", "mixed_bf16", 1, 1)]

_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from chidg_b200 import api, mesh
out = {}
for kind, prec, nt, P in json.loads(sys.argv[2]):
    pat = mesh.box_pattern(5, 4, 3, 5, mesh.nterms_of_order(P), ntime=nt)
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=41))
    b = api.ChidgVector(A, mesh.synth_vector(pat.vector_size(), seed=42))
    x = api.ChidgVector(A)
    opts = dict(tol=0.0, rtol=1e-9, nkrylov=12, inner_fgmres=0, nmax=400, precision=prec)
    if prec in ("mixed_fp32", "mixed_bf16"):
        opts.update(nkrylov=8, mixed_inner_nkrylov=10, mixed_inner_rtol=1e-2, mixed_inner_nmax=30)
    s = api.create_linear_solver("fgmres", **opts)
    s.solve(A, x, b, api.create_preconditioner(kind))
    out[f"{kind}-{prec}-{nt}-{P}"] = {"x": x.download().tolist(), "hist": s.hist.tolist(), "niter": s.niter}
print(json.dumps(out))
"""


def _run(fused):
    env = dict(os.environ, CHIDG_FUSED_MV="1" if fused else "0")
    p = subprocess.run([sys.executable, "-c", _CHILD, ROOT, json.dumps(CASES)], capture_output=True, text=True,
                       env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_fused_sweep_and_matvec_are_bitwise_the_separate_launches():
    fused, split = _run(True), _run(False)
    for key in split:
        assert fused[key]["niter"] == split[key]["niter"], key
        assert np.array_equal(np.array(fused[key]["hist"]), np.array(split[key]["hist"])), key
        assert np.array_equal(np.array(fused[key]["x"]), np.array(split[key]["x"])), key
