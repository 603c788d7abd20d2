"""Edge cases of the matrix layout against the oracle: ragged element orders
in one matrix (non-square coupling blocks), the largest block size (1024
rows), and patterns the library must refuse.

Tolerances as in tests/test_gpu_parity.py."""
import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def ragged(seed):
    base = mesh.box_pattern(3, 3, 2, 5, mesh.nterms_of_order(1))
    pat = mesh.with_element_orders(base, [(e * 7) % 3 for e in range(base.nelem)])   # P0, P1, P2 mixed
    vals = mesh.synth_values(pat, seed=seed)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(pat)
    Ag.upload(vals)
    return pat, vals, Ao, Ag


def test_ragged_matvec():
    pat, vals, Ao, Ag = ragged(101)
    x = mesh.synth_vector(Ao.n, seed=102)
    assert relerr(api.chidg_mv(Ag, api.ChidgVector(Ag, x)).download(), Ao.mv(x)) < 1e-13


@pytest.mark.parametrize("kind,schedule", [("ilu0", "stream"), ("ilu0", "tasks"), ("ilu0", "levels"), ("jacobi", "stream")])
def test_ragged_precon(kind, schedule):
    pat, vals, Ao, Ag = ragged(103)
    Mo = O.OraclePrecon(Ao, kind)
    Mo.update()
    Mg = api.create_preconditioner(kind, schedule=schedule)
    Mg.update(Ag)
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    LDg, LDo = Mg.LD(), Mo.LD()
    for k in range(pat.nblocks):
        s = slice(voff[k], voff[k] + nr[k] * nc[k])
        assert np.linalg.norm(LDg[s] - LDo[s]) <= 1e-10 * max(np.linalg.norm(LDo[s]), 1e-300), k
    v = mesh.synth_vector(Ao.n, seed=104)
    assert relerr(Mg.apply(Ag, api.ChidgVector(Ag, v)).download(), Mo.apply(v)) < 1e-11


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_ragged_fgmres(precision):
    pat, vals, Ao, Ag = ragged(105)
    b = mesh.synth_vector(Ao.n, seed=106)
    opts = dict(tol=0.0, rtol=1e-8, nkrylov=20, inner_fgmres=0, nmax=400)
    xo, ro = O.fgmres(Ao, O.OraclePrecon(Ao, "ilu0"), b, O.default_opts(**opts))
    extra = {} if precision == "fp64" else dict(nkrylov=10, mixed_inner_nkrylov=20, mixed_inner_rtol=1e-2,
                                               mixed_inner_nmax=40)
    solver = api.create_linear_solver("fgmres", **{**opts, **extra}, precision=precision)
    xg = api.ChidgVector(Ag)
    solver.solve(Ag, xg, api.ChidgVector(Ag, b), api.create_preconditioner("ilu0"))
    if precision == "fp64":
        assert solver.niter == ro["niter"]
        assert relerr(xg.download(), xo) < 1e-10
    else:
        assert solver.residual_norm <= 1.5e-8 * solver.r0norm_initial
        assert relerr(xg.download(), xo) < 1e-6


@pytest.mark.parametrize("kind", ["ilu0", "jacobi"])
def test_largest_block_size(kind):
    """1024-row blocks: the streamed matvec and sweeps at their limit, the
    diagonal inverses in panels of 8 columns."""
    pat = mesh.box_pattern(2, 1, 1, 4, 256)
    assert int(pat.bsize().max()) == 1024
    vals = mesh.synth_values(pat, seed=107)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(pat)
    Ag.upload(vals)
    x = mesh.synth_vector(Ao.n, seed=108)
    xv = api.ChidgVector(Ag, x)
    assert relerr(api.chidg_mv(Ag, xv).download(), Ao.mv(x)) < 1e-13
    Mo = O.OraclePrecon(Ao, kind)
    Mo.update()
    Mg = api.create_preconditioner(kind)
    Mg.update(Ag)
    assert relerr(Mg.apply(Ag, xv).download(), Mo.apply(x)) < 1e-10


def test_block_size_above_limit_refused():
    pat = mesh.box_pattern(2, 1, 1, 1, 1025)
    with pytest.raises(_lib.ChidgGpuError) as ei:
        api.ChidgMatrix(pat)
    assert ei.value.code == _lib.EINVAL


def test_malformed_patterns_refused():
    good = mesh.box_pattern(2, 2, 1, 1, 1, ntime=2)

    def variant(**kw):
        f = {k: getattr(good, k).copy() for k in ("elem_nvars", "elem_nterms", "elem_proc", "blk_row_elem",
                                                  "blk_row_time", "blk_col_elem", "blk_col_time", "blk_kind",
                                                  "blk_face")}
        f.update(kw)
        return mesh.BlockPattern(nelem=kw.get("nelem", good.nelem), ntime=good.ntime,
                                 **{k: v for k, v in f.items() if k != "nelem"})

    diag = np.nonzero((good.blk_row_elem == good.blk_col_elem) & (good.blk_kind == 0))[0]
    local_off = np.nonzero((good.blk_row_elem != good.blk_col_elem) & (good.blk_kind == 0))[0]
    bad_col = good.blk_col_elem.copy()
    bad_col[0] = good.nelem                                   # column element out of range
    no_diag_kind = good.blk_kind.copy()
    no_diag_kind[diag[0]] = _lib.BLK_CHIMERA                  # a row without its DIAG block
    cross_time = good.blk_col_time.copy()
    cross_time[local_off[0]] = 1 - good.blk_row_time[local_off[0]]   # LOCAL block across time levels
    zero_order = good.elem_nterms.copy()
    zero_order[1] = 0
    for pat in (variant(blk_col_elem=bad_col), variant(blk_kind=no_diag_kind), variant(blk_col_time=cross_time),
                variant(elem_nterms=zero_order)):
        with pytest.raises(_lib.ChidgGpuError) as ei:
            api.ChidgMatrix(pat)
        assert ei.value.code == _lib.EINVAL
    empty = mesh.BlockPattern(nelem=0, ntime=1, elem_nvars=np.zeros(0, np.int32), elem_nterms=np.zeros(0, np.int32),
                              elem_proc=np.zeros(0, np.int32), blk_row_elem=np.zeros(0, np.int32),
                              blk_row_time=np.zeros(0, np.int32), blk_col_elem=np.zeros(0, np.int32),
                              blk_col_time=np.zeros(0, np.int32), blk_kind=np.zeros(0, np.int32),
                              blk_face=np.zeros(0, np.int32))
    with pytest.raises(_lib.ChidgGpuError) as ei:
        api.ChidgMatrix(empty)
    assert ei.value.code == _lib.EINVAL


@pytest.mark.parametrize("nterms", [64, 100, 144])
def test_panel_inverse_block_sizes(nterms):
    """320-, 500- and 720-row blocks (P3 and wider): the diagonal inverses run
    in panels of 32, 16 and 8 columns; the factors and z = M v against the
    oracle (factor blocks within 1e-10 of the block norm)."""
    pat = mesh.box_pattern(3, 2, 1, 5, nterms)
    vals = mesh.synth_values(pat, seed=111)
    Ao = O.OracleMatrix(pat)
    Ao.set_values(vals)
    Ag = api.ChidgMatrix(pat)
    Ag.upload(vals)
    Mo = O.OraclePrecon(Ao, "ilu0")
    Mo.update()
    Mg = api.create_preconditioner("ilu0")
    Mg.update(Ag)
    ldo, ldg = Mo.LD(), Mg.LD()
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    for k in range(pat.nblocks):
        if pat.blk_col_elem[k] > pat.blk_row_elem[k]:
            continue                                     # U blocks are A's
        a, g = ldo[voff[k]:voff[k] + nr[k] * nc[k]], ldg[voff[k]:voff[k] + nr[k] * nc[k]]
        assert np.abs(a - g).max() <= 1e-10 * np.abs(a).max(), k
    x = mesh.synth_vector(Ao.n, seed=112)
    assert relerr(Mg.apply(Ag, api.ChidgVector(Ag, x)).download(), Mo.apply(x)) < 1e-10
