"""The mixed-precision factorisation's block products on the tcgen05 tensor
cores (k_task_gemm_umma: TF32 operands, FP32 accumulation in tensor memory).

Its FP32 factors are checked against the FP64 factors (TF32 rounding bound)
and against the same products by the mma.sync TF32 kernel, computed in a
child process (CHIDG_FACTOR32_MMA=sync): both round the operands to TF32 the
same way and accumulate K in the same steps of 8 in FP32, and they give the
same factors bit for bit."""
import os
import subprocess
import sys

import numpy as np
import pytest

from chidg_b200 import api, mesh

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# (box, order, fields): 40-row blocks (one M tile), 135 (two), 144 (the largest)
CASES = [((4, 3, 3), 1, 5), ((3, 3, 2), 2, 5), ((3, 2, 2), 1, 18)]


def factors(shape, P, nvars, precision):
    pat = mesh.box_pattern(*shape, nvars, mesh.nterms_of_order(P))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=51))
    M = api.create_preconditioner("ilu0")
    M.update(A, precision=precision)
    return pat, (M.LD32() if precision != "fp64" else M.LD())


CHILD = """
import sys, numpy as np
sys.path.insert(0, {root!r})
from tests.test_gpu_umma import factors
pat, ld = factors({shape!r}, {P!r}, {nvars!r}, "mixed_fp32")
np.save({out!r}, ld)
"""


@pytest.mark.parametrize("shape,P,nvars", CASES)
def test_tcgen05_factor_products(shape, P, nvars, tmp_path):
    pat, ld32 = factors(shape, P, nvars, "mixed_fp32")
    _, ld64 = factors(shape, P, nvars, "fp64")
    out = str(tmp_path / "sync.npy")
    env = dict(os.environ, CHIDG_FACTOR32_MMA="sync")
    subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, shape=shape, P=P, nvars=nvars, out=out)],
                   check=True, env=env, timeout=600)
    ld_sync = np.load(out)
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    worst64 = worst_sync = 0.0
    for k in range(pat.nblocks):
        a = ld64[voff[k]:voff[k] + nr[k] * nc[k]]
        if not np.any(a):
            continue
        g = ld32[voff[k]:voff[k] + nr[k] * nc[k]].astype(np.float64)
        s = ld_sync[voff[k]:voff[k] + nr[k] * nc[k]].astype(np.float64)
        worst64 = max(worst64, np.linalg.norm(g - a) / np.linalg.norm(a))
        worst_sync = max(worst_sync, np.linalg.norm(g - s) / np.linalg.norm(s))
    assert np.all(np.isfinite(ld32))
    assert worst64 < 5e-3, worst64          # TF32 operands (11-bit significands)
    assert worst_sync == 0.0 and np.array_equal(ld32, ld_sync), worst_sync


def test_download_ld32_refused_after_fp64_update():
    pat = mesh.box_pattern(2, 2, 2, 5, mesh.nterms_of_order(1))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=52))
    M = api.create_preconditioner("ilu0")
    M.update(A)
    with pytest.raises(api.ChidgGpuError):
        M.LD32()
