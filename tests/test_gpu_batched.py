"""Batched FGMRES: independent systems of different sizes and block sizes,
packed block-diagonally and solved together, each matching its own oracle
solve (same iteration count, residual history within 1e-8 relative, solution
within 1e-10 relative)."""
import numpy as np
import pytest

from chidg_b200 import api, mesh
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SYSTEMS = [((3, 3, 2), 1, 11), ((2, 2, 2), 2, 12), ((4, 2, 2), 1, 13), ((2, 2, 1), 0, 14), ((3, 2, 2), 2, 15)]


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def build():
    pats, vals, rhs = [], [], []
    for shape, P, seed in SYSTEMS:
        p = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P))
        pats.append(p)
        vals.append(mesh.synth_values(p, seed=seed))
        rhs.append(mesh.synth_vector(p.vector_size(), seed=seed + 100))
    union, sys_elem = mesh.concat_patterns(pats)
    return pats, vals, rhs, union, sys_elem


@pytest.mark.parametrize("prec", ["ilu0", "jacobi"])
def test_batched_matches_individual_oracle_solves(prec):
    pats, vals, rhs, union, sys_elem = build()
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=300)
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    solver = api.create_linear_solver("fgmres", **opts)
    res = solver.solve_batched(A, x, b, api.create_preconditioner(prec), sys_elem)
    xg = x.download()
    off = 0
    for s, (pat, v, r) in enumerate(zip(pats, vals, rhs)):
        Ao = O.OracleMatrix(pat)
        Ao.set_values(v)
        xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, prec), r, O.default_opts(**opts))
        n = pat.vector_size()
        assert res[s]["niter"] == ro["niter"], (s, res[s]["niter"], ro["niter"])
        assert relerr(res[s]["hist"], ro["hist"]) < 1e-8
        assert relerr(xg[off:off + n], xo) < 1e-10
        assert res[s]["residual_norm"] == pytest.approx(ro["residual_norm"], rel=1e-6)
        off += n


def test_batched_zero_rhs_system():
    pats, vals, rhs, union, sys_elem = build()
    rhs[1][:] = 0.0
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    solver = api.create_linear_solver("fgmres", tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=300)
    res = solver.solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
    eo = union.elem_offsets()
    xs = x.download()[eo[sys_elem[1]]:eo[sys_elem[2]]]
    assert res[1]["niter"] == 0 and np.all(xs == 0.0)
    assert all(r["residual_norm"] <= 2e-8 * max(r["r0norm_initial"], 1e-300) for i, r in enumerate(res) if i != 1)


def test_batched_fp32_preconditioner_matches_single_solves():
    """FP64 Krylov with FP32 preconditioner blocks, batched: every system
    reaches the FP64 residual target and agrees with its FP64 oracle solve."""
    pats, vals, rhs, union, sys_elem = build()
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=300, precision="mixed_precon_fp32")
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    res = api.create_linear_solver("fgmres", **opts).solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
    xb = x.download()
    eo = union.elem_offsets()
    for s, (p, v, r) in enumerate(zip(pats, vals, rhs)):
        assert res[s]["residual_norm"] <= 1.5e-8 * res[s]["r0norm_initial"]
        Ao = O.OracleMatrix(p)
        Ao.set_values(v)
        xo, _ = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), r, O.default_opts(tol=0.0, rtol=1e-10, nkrylov=30,
                                                                           inner_fgmres=0, nmax=300))
        assert relerr(xb[eo[sys_elem[s]]:eo[sys_elem[s + 1]]], xo) < 1e-6


@pytest.mark.parametrize("prec", ["mixed_fp32", "mixed_bf16"])
def test_batched_fp32_inner_solves_reach_fp64_accuracy(prec):
    """FP64 outer FGMRES whose every step is preconditioned by a batched FP32
    inner FGMRES (FP32 or BF16 factors and copy of A): every system reaches
    the FP64 residual target, its inner iterations are counted, and x agrees
    with the system's FP64 oracle solve."""
    pats, vals, rhs, union, sys_elem = build()
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=8, inner_fgmres=0, nmax=300, precision=prec,
                mixed_inner_nkrylov=10, mixed_inner_rtol=1e-2, mixed_inner_nmax=30)
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    res = api.create_linear_solver("fgmres", **opts).solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
    xb = x.download()
    eo = union.elem_offsets()
    for s, (p, v, r) in enumerate(zip(pats, vals, rhs)):
        assert res[s]["residual_norm"] <= 1.5e-8 * res[s]["r0norm_initial"], (s, res[s])
        assert res[s]["inner_iters"] >= res[s]["niter"] > 0, (s, res[s])
        Ao = O.OracleMatrix(p)
        Ao.set_values(v)
        xo, _ = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), r, O.default_opts(tol=0.0, rtol=1e-10, nkrylov=30,
                                                                           inner_fgmres=0, nmax=300))
        assert relerr(xb[eo[sys_elem[s]]:eo[sys_elem[s + 1]]], xo) < 1e-6


def test_batched_harmonic_balance_systems():
    """Systems with 3 coupled time levels (harmonic-balance blocks), batched:
    each matches its own FP64 oracle solve."""
    pats, vals, rhs = [], [], []
    for shape, seed in [((2, 2, 2), 41), ((3, 2, 1), 42), ((2, 1, 2), 43)]:
        p = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(1), ntime=3)
        pats.append(p)
        vals.append(mesh.synth_values(p, seed=seed))
        rhs.append(mesh.synth_vector(p.vector_size(), seed=seed + 100))
    union, sys_elem = mesh.concat_patterns(pats)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=10, inner_fgmres=0, nmax=300)
    A = api.ChidgMatrix(union)
    A.upload(np.concatenate(vals))
    b = api.ChidgVector(A, np.concatenate(rhs))
    x = api.ChidgVector(A)
    res = api.create_linear_solver("fgmres", **opts).solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
    xb = x.download()
    eo = union.elem_offsets()
    for s, (p, v, r) in enumerate(zip(pats, vals, rhs)):
        Ao = O.OracleMatrix(p)
        Ao.set_values(v)
        xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), r, O.default_opts(**opts))
        assert res[s]["niter"] == ro["niter"]
        assert relerr(xb[eo[sys_elem[s]]:eo[sys_elem[s + 1]]], xo) < 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_batched_graph_replay_matches_eager_solves(precision):
    """The same batch structure solved again (new values, the next Newton
    step) replays its Arnoldi steps from captured graphs: the second and later
    calls give bitwise the result an eager solve of the same values gives
    (CHIDG_BATCH_GRAPHS=0 in a process of its own), restarts included.  With
    FP32 inner solves it is the inner solves' steps that are replayed (an
    outer step runs the inner solve's host loop), captured at the second
    inner solve of the first call."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    child = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from chidg_b200 import api, mesh
pats = [mesh.box_pattern(*s, 5, mesh.nterms_of_order(P)) for s, P in (((3, 3, 2), 1), ((2, 2, 2), 2), ((4, 2, 2), 1))]
union, sys_elem = mesh.concat_patterns(pats)
A = api.ChidgMatrix(union)
b = api.ChidgVector(A, mesh.synth_vector(union.vector_size(), seed=7))
x = api.ChidgVector(A)
M = api.create_preconditioner("ilu0")
opts = dict(tol=0.0, rtol=1e-9, nkrylov=6, inner_fgmres=0, nmax=300, precision=sys.argv[2])
if sys.argv[2] != "fp64":
    opts.update(nkrylov=3, mixed_inner_nkrylov=4, mixed_inner_rtol=1e-2, mixed_inner_nmax=12)
solver = api.create_linear_solver("fgmres", **opts)
out = []
for step in range(4):
    A.upload(mesh.synth_values(union, seed=20 + step))
    res = solver.solve_batched(A, x, b, M, sys_elem)
    out.append({"x": x.download().tolist(), "niter": [r["niter"] for r in res], "inner": [r["inner_iters"] for r in res],
                "hist": [r["hist"].tolist() for r in res], "res": [r["residual_norm"] for r in res]})
print(json.dumps(out))
"""

    def run(graphs):
        env = dict(os.environ, CHIDG_BATCH_GRAPHS="1" if graphs else "0")
        p = subprocess.run([sys.executable, "-c", child, root, precision], capture_output=True, text=True, env=env,
                           timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        return json.loads(p.stdout.strip().splitlines()[-1])

    g, e = run(True), run(False)
    for step in range(4):
        assert g[step]["niter"] == e[step]["niter"], step
        assert g[step]["inner"] == e[step]["inner"], step
        if precision == "fp64":
            assert max(g[step]["niter"]) > 6        # restarts happen
        else:
            assert max(g[step]["inner"]) > 4        # inner restarts happen
        assert g[step]["hist"] == e[step]["hist"], step
        assert np.array_equal(np.array(g[step]["x"]), np.array(e[step]["x"])), step


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_skipping_frozen_systems_changes_no_answer(precision):
    """While a batched Arnoldi step runs, the streamed sweeps and matvecs skip
    the rows of systems that have already converged.  Systems of uneven
    difficulty (they converge at different steps) give bitwise the same
    iterations, histories and solutions as a process that runs every row
    (CHIDG_BATCH_SKIP_FROZEN=0)."""
    import json
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    child = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from chidg_b200 import api, mesh
shapes = [((4, 3, 3), 1, 1.0), ((2, 2, 2), 2, 0.05), ((3, 3, 2), 2, 1.0), ((2, 2, 1), 1, 0.02), ((3, 2, 2), 1, 0.5)]
pats, vals = [], []
for k, (shape, P, off) in enumerate(shapes):
    p = mesh.box_pattern(*shape, 5, mesh.nterms_of_order(P))
    v = mesh.synth_values(p, seed=60 + k)
    # scale the off-diagonal blocks: weakly coupled systems converge in fewer steps
    ro, nval = p.value_offsets()
    nr, nc = p.block_dims()
    for i in range(p.nblocks):
        if p.blk_row_elem[i] != p.blk_col_elem[i]:
            v[ro[i]:ro[i] + nr[i] * nc[i]] *= off
    pats.append(p)
    vals.append(v)
union, sys_elem = mesh.concat_patterns(pats)
A = api.ChidgMatrix(union)
A.upload(np.concatenate(vals))
b = api.ChidgVector(A, mesh.synth_vector(union.vector_size(), seed=9))
x = api.ChidgVector(A)
opts = dict(tol=0.0, rtol=1e-9, nkrylov=8, inner_fgmres=0, nmax=300, precision=sys.argv[2])
if sys.argv[2] != "fp64":
    opts.update(nkrylov=4, mixed_inner_nkrylov=6, mixed_inner_rtol=1e-2, mixed_inner_nmax=12)
res = api.create_linear_solver("fgmres", **opts).solve_batched(A, x, b, api.create_preconditioner("ilu0"), sys_elem)
print(json.dumps({"x": x.download().tolist(), "niter": [r["niter"] for r in res], "inner": [r["inner_iters"] for r in res],
                  "hist": [r["hist"].tolist() for r in res], "res": [r["residual_norm"] for r in res]}))
"""

    def run(skip):
        env = dict(os.environ, CHIDG_BATCH_SKIP_FROZEN="1" if skip else "0")
        p = subprocess.run([sys.executable, "-c", child, root, precision], capture_output=True, text=True, env=env,
                           timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        return json.loads(p.stdout.strip().splitlines()[-1])

    s, a = run(True), run(False)
    assert len(set(a["niter"])) > 1                 # the systems converge at different steps
    assert s["niter"] == a["niter"] and s["inner"] == a["inner"]
    assert s["hist"] == a["hist"]
    assert s["res"] == a["res"]
    assert np.array_equal(np.array(s["x"]), np.array(a["x"]))
