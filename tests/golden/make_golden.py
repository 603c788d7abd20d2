"""Regenerate tests/golden/reference_kat.json from the reference's own unit
tests, read as text (the reference cannot be compiled here: no Fortran
compiler).  Each known-answer test poke-sets matrix blocks with
`...lblks(ielem,itime)%loc(1,K,itime)` / `%data_(imat)%mat = VALUE`, sets the
right-hand side per element, and asserts values; this script replays that
bookkeeping and records the matrices, right-hand sides and expected values.

Usage: python tests/golden/make_golden.py [/path/to/ChiDG]   (default /root/reference)
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
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kat.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
