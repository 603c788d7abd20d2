"""Regenerate tests/golden/reference_kat.json from the reference's own unit
tests, read as text (the reference cannot be compiled here: no Fortran
compiler).  Each known-answer test poke-sets matrix blocks with
`...lblks(ielem,itime)%loc(1,K,itime)` / `%data_(imat)%mat = VALUE`, sets the
right-hand side per element, and asserts values; this script replays that
bookkeeping and records the matrices, right-hand sides and expected values.

Usage: python tests/golden/make_golden.py /path/to/ChiDG
(the root of the ChiDG source tree; required)
"""
from __future__ import annotations

import json
import os
import re
import sys

CONST = {"ZERO": 0.0, "ONE": 1.0, "TWO": 2.0, "THREE": 3.0, "FOUR": 4.0, "FIVE": 5.0, "SIX": 6.0,
         "SEVEN": 7.0, "EIGHT": 8.0, "NINE": 9.0, "TEN": 10.0}

TESTS = {
    # name: (file, nelem_xi, ntime)
    "ilu0": ("test/unit_testing/preconditioners/test_ILU0_mod.pf", 3, 1),
    "ilu0_hb": ("test/unit_testing/preconditioners/test_ILU0_HB_mod.pf", 3, 3),
    "fgmres": ("test/unit_testing/linear_solvers/test_fgmres.pf", 3, 1),
    "fgmres_ref": ("test/unit_testing/linear_solvers/test_fgmres_ref.pf", 2, 1),
}


def value(expr: str) -> float:
    expr = expr.strip()
    sign = 1.0
    if expr.startswith("-"):
        sign, expr = -1.0, expr[1:].strip()
    expr = expr.replace("_rk", "")
    if expr in CONST:
        return sign * CONST[expr]
    if expr.startswith("(") and expr.endswith(")"):
        inner = expr[1:-1]
        m = re.fullmatch(r"\s*(\w+)\s*/\s*([\d.]+)\s*", inner)
        if m:
            return sign * value(m.group(1)) / float(m.group(2))
    return sign * float(expr)


def parse(path: str):
    text = open(path).read().splitlines()
    state = {"ielem": None, "itime": None, "idomain": 1}
    locvar = {}
    blocks = {}      # (elem, time, col_elem) -> value
    rhs = {}         # elem -> value
    asserts = []     # (kind, elem or (elem, col), value)
    solver_tol = None
    tol = None
    pending_col = None
    for raw in text:
        line = raw.split("!")[0].strip()
        if not line:
            continue
        m = re.fullmatch(r"(ielem|itime|idomain)\s*=\s*(\d+)", line)
        if m:
            state[m.group(1)] = int(m.group(2))
            continue
        m = re.fullmatch(r"(?:real\(rk\)\s*::\s*)?tol\s*=\s*([\d.eE+-]+)_rk", line)
        if m:
            tol = float(m.group(1))
            continue
        m = re.search(r"linear_solver%tol\s*=\s*([\d.eE+-]+)_rk", line)
        if m:
            solver_tol = float(m.group(1))
            continue
        resolve = lambda s: state[s] if s in state else int(s)
        m = re.search(r"imat\s*=\s*self%ILU0%LD%dom\(1\)%lblks\(ielem,\s*itime\)%loc\(1,\s*(\d+),", line)
        if m:
            pending_col = int(m.group(1))
            continue
        m = re.search(r"(\w+)\s*=\s*[\w%()]*lblks\((\w+),\s*(\w+)\)%loc\(\s*1\s*,\s*(\d+)\s*,", line)
        if m:
            locvar[m.group(1)] = (resolve(m.group(2)), resolve(m.group(3)), int(m.group(4)))
            continue
        m = re.search(r"(?<!ILU0%LD%)dom\(1\)%lblks\((\w+),\s*(\w+)\)%data_\((\w+)\)%mat\s*=\s*(.+)$", line)
        if m and "ILU0" not in line:
            e, t, col = locvar[m.group(3)]
            blocks[(e, t, col)] = value(m.group(4))
            continue
        m = re.search(r"rhs%dom\(1\)%vecs\((\d+)\)%vec\s*=\s*(.+)$", line) or \
            re.fullmatch(r"b%dom\(1\)%vecs\((\d+)\)%vec\s*=\s*(.+)", line)
        if m:
            rhs[int(m.group(1))] = value(m.group(2))
            continue
        m = re.search(r"@assertEqual\((.+?),\s*self%ILU0%LD%dom\(1\)%lblks\(ielem,\s*itime\)%data_\(imat\)%mat\(1,1\)\)", line)
        if m:
            asserts.append(("LD", [state["ielem"], state["itime"], pending_col], value(m.group(1))))
            continue
        m = re.search(r"@assertEqual\((.+?),\s*z%dom\(1\)%vecs\((\d+)\)%vec\((?:itime_)?(\d+)\),\s*tol\)", line)
        if m:
            # entry index inside the element vector; with one mode and one field it
            # is the time level (get_time_start(itime) = itime)
            asserts.append(("z", [int(m.group(2)), int(m.group(3))], value(m.group(1))))
            continue
        m = re.search(r"@assertEqual\((.+?),\s*x%dom\(1\)%vecs\((\d+)\)%vec,\s*tol\)", line)
        if m:
            asserts.append(("x", [int(m.group(2)), 1], value(m.group(1))))
            continue
    return blocks, rhs, asserts, tol, solver_tol


# Operator known-answer tests: two 2x2x2 domains, one field, P1 (8 modes).
# Each test sets some blocks to a constant (or to M(i,j) = i), sets x per
# element, multiplies and asserts whole element segments of the result.
OPERATOR_TESTS = {
    # name: (file, subroutine)
    "mv": ("test/unit_testing/containers/test_chidg_matrix_operator_mv.pf", "test_chidg_matrix_operator_mv"),
    "mtv": ("test/unit_testing/containers/test_chidg_matrix_operator_mtv.pf", "test_chidg_matrix_operator_mtv"),
    "mtv_2": ("test/unit_testing/containers/test_chidg_matrix_operator_mtv.pf", "test_chidg_matrix_operator_mtv_2"),
}
OP_ELEMS_PER_DOMAIN, OP_NTERMS = 8, 8
# Chimera donors of the "D2 E8 M1 : Overlapping : NonMatching" mesh, used by
# the tests that address blocks through chi_blks(...)%dparent_g/eparent_g(k)
# instead of loc(dom, elem).  The mesh's hole cutting is not reproducible
# here; the donors follow from test_chidg_matrix_operator_mtv's own asserts
# (b(2,1) = 2*0.1*nterms and b(2,3) = 3*0.1*nterms: the two donors of domain 1
# element 2 are domain 2 elements 1 and 3; b(1,2) = 4*0.2*nterms: the donor of
# domain 2 element 1 is domain 1 element 2).  (domain, element) -> donors.
CHIMERA_DONORS = {(1, 2): [(2, 1), (2, 3)], (2, 1): [(1, 2)]}


def op_value(expr: str) -> float:
    """bref_* expressions: products and sums of literals, named constants and nterms_s."""
    e = expr.replace("_rk", "")
    e = re.sub(r"\bnterms_s\b", str(OP_NTERMS), e)
    for k, v in CONST.items():
        e = re.sub(rf"\b{k}\b", repr(v), e)
    if not re.fullmatch(r"[\d.+*/() \-]+", e):
        raise ValueError(f"unsupported expression {expr!r}")
    return float(eval(e, {"__builtins__": {}}))   # arithmetic on literals only


def parse_operator(path: str, subroutine: str):
    text = open(path).read()
    m = re.search(rf"subroutine {subroutine}\(\)(.*?)end subroutine {subroutine}", text, re.S)
    body = m.group(1)
    state = {"idom": None, "ielem": None, "itime": 1}
    locvar, blocks, x, bref, asserts = {}, {}, {}, {}, []
    mode, tol, rowindex = None, None, False
    gid = lambda d, e: (d - 1) * OP_ELEMS_PER_DOMAIN + (e - 1)     # 0-based global element
    res = lambda tok: state[tok] if tok in state else int(tok)
    for raw in body.splitlines():
        line = raw.split("!")[0].strip()
        if not line:
            continue
        if (m := re.fullmatch(r"(idom|ielem|itime)\s*=\s*(\d+)", line)):
            state[m.group(1)] = int(m.group(2))
        elif (m := re.fullmatch(r"tol\s*=\s*([\d.eE+-]+)_rk", line)):
            tol = float(m.group(1))
        elif (m := re.fullmatch(r"(\w+)\s*=\s*A%dom\((\w+)\)%(lblks|chi_blks)\(ielem,\s*itime\)%loc\((\d+),\s*(\d+),\s*itime\)", line)):
            kind = 0 if m.group(3) == "lblks" else 1
            locvar[m.group(1)] = (kind, gid(res(m.group(2)), state["ielem"]), gid(int(m.group(4)), int(m.group(5))))
        elif (m := re.fullmatch(r"(idom_d|ielem_d)\s*=\s*A%dom\((\w+)\)%chi_blks\(ielem,\s*itime\)%(dparent_g|eparent_g)\((\d+)\)", line)):
            donor = CHIMERA_DONORS[(res(m.group(2)), state["ielem"])][int(m.group(4)) - 1]
            state[m.group(1)] = donor[0] if m.group(3) == "dparent_g" else donor[1]
        elif (m := re.fullmatch(r"M\(i,j\)\s*=\s*real\(i,\s*rk\)", line)):
            rowindex = True
        elif (m := re.fullmatch(r"A%dom\((\w+)\)%(lblks|chi_blks)\(ielem,\s*itime\)%data_\((\w+)\)%mat\s*=\s*(\w+)", line)):
            dom = res(m.group(1))
            if m.group(3) in locvar:
                key = locvar[m.group(3)]
            else:                                   # chi_blks%data_(k): the k-th donor
                d, e = CHIMERA_DONORS[(dom, state["ielem"])][int(m.group(3)) - 1]
                key = (1, gid(dom, state["ielem"]), gid(d, e))
            if m.group(4) == "M":
                assert rowindex
                blocks[key] = "rowindex"
            else:
                blocks[key] = CONST[m.group(4)]
        elif (m := re.fullmatch(r"x%dom\((\w+)\)%vecs\((\w+)\)%vec\s*=\s*([\d.]+)_rk", line)):
            x[gid(res(m.group(1)), res(m.group(2)))] = float(m.group(3))
        elif (m := re.fullmatch(r"b\s*=\s*(chidg_mv|transposed_matrix_vector_product)\(A,\s*x\)", line)):
            mode = "mv" if m.group(1) == "chidg_mv" else "mtv"
        elif (m := re.fullmatch(r"(bref_\w+)\s*=\s*(.+)", line)):
            bref[m.group(1)] = op_value(m.group(2))
        elif (m := re.fullmatch(r"@assertEqual\((bref_\w+),\s*b%dom\((\d+)\)%vecs\((\d+)\)%vec,\s*tol\)", line)):
            asserts.append([gid(int(m.group(2)), int(m.group(3))), bref[m.group(1)]])
    assert mode and asserts and tol
    return {"subroutine": subroutine, "mode": mode, "nelem": 2 * OP_ELEMS_PER_DOMAIN, "nvars": 1,
            "nterms": OP_NTERMS, "tol": tol,
            # [row element, column element, kind (0 LOCAL, 1 CHIMERA), value or "rowindex" (M(i,j) = i)]
            "blocks": [[r, c, k, v] for (k, r, c), v in sorted(blocks.items())],
            "x": [[e, v] for e, v in sorted(x.items())],
            "asserts": asserts}


def main(root: str):
    out = {"source": "ChiDG unit tests (read as text by tests/golden/make_golden.py)", "cases": {}}
    for name, (rel, nx, ntime) in TESTS.items():
        blocks, rhs, asserts, tol, solver_tol = parse(os.path.join(root, rel))
        out["cases"][name] = {
            "file": rel, "nelem_xi": nx, "ntime": ntime,
            # 1-based element ids as in the reference; col_elem = eparent_g of the block
            "blocks": [[e, t, c, v] for (e, t, c), v in sorted(blocks.items())],
            "rhs": [[e, v] for e, v in sorted(rhs.items())],
            "asserts": [[k, idx, v] for k, idx, v in asserts],
            "tol": tol, "solver_tol": solver_tol,
        }
    for name, (rel, sub) in OPERATOR_TESTS.items():
        out["cases"][name] = {"file": rel, **parse_operator(os.path.join(root, rel), sub)}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kat.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/ChiDG")
    main(sys.argv[1])
