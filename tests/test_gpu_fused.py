"""The matvec rows run inside the streamed backward sweep (the fused pass that
FGMRES takes for z = M v followed by w = A z) agree with the separate launches
to rounding: the fused rows stream the diagonal and lower blocks and add the
sweep's products of the upper blocks with z (the U partials the sweep formed),
where the separate matvec sums every block of the row in one pass, and the
launches' stages differ in size, so the chunk boundaries of the partial sums
differ too.  Checked on whole FGMRES solves against a process that runs the
separate launches (CHIDG_FUSED_MV=0), and against a process whose fused rows
stream every block (CHIDG_FUSED_REUSE=0):
FP64 and FP32 preconditioner blocks take the same iterations with the residual
history within 1e-10 and x within 1e-12; the FP32 and BF16 inner solves reach
the same FP64 residual with x within 1e-6.  ILU0 and Jacobi, one and three
time levels."""
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
    out[f"{kind}-{prec}-{nt}-{P}"] = {"x": x.download().tolist(), "hist": s.hist.tolist(), "niter": s.niter,
                                      "rel_res": s.residual_norm / s.r0norm_initial}
print(json.dumps(out))
"""


def _run(fused, reuse=True):
    env = dict(os.environ, CHIDG_FUSED_MV="1" if fused else "0", CHIDG_FUSED_REUSE="1" if reuse else "0")
    p = subprocess.run([sys.executable, "-c", _CHILD, ROOT, json.dumps(CASES)], capture_output=True, text=True,
                       env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _agree(f, s, key):
    if "mixed_fp32" in key or "mixed_bf16" in key:
        assert f["rel_res"] <= 1e-9 * 1.0001 and s["rel_res"] <= 1e-9 * 1.0001, key
        assert relerr(f["x"], s["x"]) <= 1e-6, key
        return
    assert f["niter"] == s["niter"], key
    assert relerr(f["hist"], s["hist"]) <= 1e-10, key
    assert relerr(f["x"], s["x"]) <= 1e-12, key


def test_fused_sweep_and_matvec_agree_with_the_separate_launches():
    fused, whole, split = _run(True), _run(True, reuse=False), _run(False)
    for key in split:
        _agree(fused[key], split[key], key)
        _agree(whole[key], split[key], key)
        _agree(fused[key], whole[key], key)
