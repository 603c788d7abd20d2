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
