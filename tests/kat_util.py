"""Known-answer systems of the reference's unit tests (tests/golden/reference_kat.json)."""
import json
import os

import numpy as np

from chidg_b200 import mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_kat.json")


def load_cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def build(case):
    """Pattern, packed block values and right-hand side of a KAT (P0 scalar, 1x1 blocks)."""
    pat = mesh.box_pattern(case["nelem_xi"], 1, 1, 1, 1, ntime=case["ntime"])
    voff, nval = pat.value_offsets()
    vals = np.zeros(nval)
    table = {(e - 1, t - 1, c - 1): v for e, t, c, v in case["blocks"]}
    for k in range(pat.nblocks):
        if pat.blk_kind[k] != 0:
            continue
        key = (int(pat.blk_row_elem[k]), int(pat.blk_row_time[k]), int(pat.blk_col_elem[k]))
        vals[voff[k]] = table.get(key, 0.0)
    b = np.zeros(pat.vector_size())
    eo = pat.elem_offsets()
    for e, v in case["rhs"]:
        b[eo[e - 1]:eo[e]] = v
    return pat, vals, b


def ld_index(pat, e, t, c):
    """Packed position of LOCAL block (row e, time t, column c), 1-based ids as in the tests."""
    voff, _ = pat.value_offsets()
    for k in range(pat.nblocks):
        if (pat.blk_kind[k] == 0 and pat.blk_row_elem[k] == e - 1 and pat.blk_row_time[k] == t - 1
                and pat.blk_col_elem[k] == c - 1):
            return voff[k]
    raise KeyError((e, t, c))


def build_operator(case, order="reference"):
    """Pattern, packed values and x of an operator KAT (mv / mtv): one field,
    `nterms` modes, a DIAG block on every element plus the blocks the test sets;
    a block is a constant or M(i,j) = i (1-based row index).  Blocks are listed
    per row in the reference's storage order (lblks, then chi_blks), or with
    order="by_column" by column element whatever their kind."""
    E, nt = case["nelem"], case["nterms"]
    listed = {(r, c, k): v for r, c, k, v in case["blocks"]}
    blocks = [(e, e, 0) for e in range(E) if (e, e, 0) not in listed] + list(listed)
    if order == "reference":
        blocks.sort(key=lambda t: (t[0], t[2], t[1]))
    else:
        blocks.sort()
    i32 = lambda a: np.asarray(a, dtype=np.int32)
    pat = mesh.BlockPattern(
        nelem=E, ntime=1, elem_nvars=i32([case["nvars"]] * E), elem_nterms=i32([nt] * E), elem_proc=i32([0] * E),
        blk_row_elem=i32([r for r, _, _ in blocks]), blk_row_time=i32([0] * len(blocks)),
        blk_col_elem=i32([c for _, c, _ in blocks]), blk_col_time=i32([0] * len(blocks)),
        blk_kind=i32([k for _, _, k in blocks]),
        blk_face=i32([mesh.DIAG if r == c else mesh.OTHER for r, c, _ in blocks]))
    voff, nval = pat.value_offsets()
    nr, nc = pat.block_dims()
    vals = np.zeros(nval)
    for k, key in enumerate(blocks):
        v = listed.get(key, 0.0)
        if v == "rowindex":
            blk = np.repeat(np.arange(1, nr[k] + 1, dtype=np.float64)[:, None], nc[k], axis=1)
        else:
            blk = np.full((nr[k], nc[k]), float(v))
        vals[voff[k]:voff[k] + nr[k] * nc[k]] = blk.ravel(order="F")
    x = np.zeros(pat.vector_size())
    eo = pat.elem_offsets()
    for e, v in case["x"]:
        x[eo[e]:eo[e + 1]] = v
    return pat, vals, x
