"""ctypes wrapper of the CPU FP64 oracle (oracle/libchidg_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker.  The product
(chidg_b200) never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchidg_oracle.so")

I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)
DP = C.POINTER(C.c_double)
VP = C.c_void_p

IDENTITY, JACOBI, ILU0, RASILU0, HB = 0, 1, 2, 3, 4
PRECON_NAMES = {"identity": IDENTITY, "jacobi": JACOBI, "ilu0": ILU0, "rasilu0": RASILU0, "hb": HB}


class Opts(C.Structure):
    _fields_ = [("tol", C.c_double), ("rtol", C.c_double), ("nmax", C.c_int32), ("nkrylov", C.c_int32),
                ("orthogonalization", C.c_int32), ("inner_fgmres", C.c_int32), ("inner_tol", C.c_double),
                ("inner_rtol", C.c_double), ("inner_nmax", C.c_int32), ("inner_nkrylov", C.c_int32),
                ("inner_orthogonalization", C.c_int32), ("use_controller", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("niter", C.c_int32), ("nrestart", C.c_int32), ("residual_norm", C.c_double),
                ("res_estimate", C.c_double), ("r0norm_initial", C.c_double), ("nhist", C.c_int32)]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_matrix_create.restype = VP
        L.orc_matrix_create.argtypes = [C.c_int32, C.c_int32, I32P, I32P, I32P, C.c_int64, I32P, I32P, I32P, I32P, I32P]
        L.orc_matrix_destroy.argtypes = [VP]
        L.orc_matrix_nvalues.restype = C.c_int64
        L.orc_matrix_nvalues.argtypes = [VP]
        L.orc_matrix_nvec.restype = C.c_int64
        L.orc_matrix_nvec.argtypes = [VP]
        for f in ("orc_matrix_set_values", "orc_matrix_get_values"):
            getattr(L, f).argtypes = [VP, DP]
        L.orc_matrix_touch.argtypes = [VP]
        L.orc_matrix_set_transposed.argtypes = [VP, C.c_int32]
        L.orc_mv.argtypes = [VP, DP, DP]
        L.orc_dot.restype = C.c_double
        L.orc_dot.argtypes = [VP, DP, DP]
        L.orc_norm.restype = C.c_double
        L.orc_norm.argtypes = [VP, DP]
        L.orc_inv.argtypes = [C.c_int32, DP, DP]
        L.orc_set_threads.argtypes = [C.c_int32]
        L.orc_get_threads.restype = C.c_int32
        L.orc_precon_create.restype = VP
        L.orc_precon_create.argtypes = [VP, C.c_int32]
        L.orc_precon_destroy.argtypes = [VP]
        L.orc_precon_update.argtypes = [VP, VP]
        L.orc_precon_apply.argtypes = [VP, VP, DP, DP]
        L.orc_precon_error_elem.argtypes = [VP]
        L.orc_precon_get_LD.argtypes = [VP, DP]
        L.orc_fgmres_solve.argtypes = [VP, VP, DP, DP, C.POINTER(Opts), C.POINTER(Result), DP, C.c_int32]
        _L = L
    return _L


def set_threads(n: int) -> None:
    """Host threads of the oracle's data-parallel loops (results are bitwise
    the same for every count)."""
    if lib().orc_set_threads(int(n)):
        raise ValueError("oracle: thread count must be >= 1")


def get_threads() -> int:
    return int(lib().orc_get_threads())


def _dp(a):
    return a.ctypes.data_as(DP)


def default_opts(**kw) -> Opts:
    """linear_solver_t defaults (src/linear_solvers/type_linear_solver.f90:23-40)."""
    o = Opts(tol=1e-8, rtol=1e-10, nmax=-1, nkrylov=2000, orthogonalization=0, inner_fgmres=1, inner_tol=0.1,
             inner_rtol=0.1, inner_nmax=100, inner_nkrylov=100, inner_orthogonalization=0, use_controller=0)
    for k, v in kw.items():
        if k in ("orthogonalization", "inner_orthogonalization") and isinstance(v, str):
            v = 0 if v.upper() == "CGS" else 1
        setattr(o, k, int(v) if isinstance(v, bool) else v)
    return o


class OracleMatrix:
    """chidg_matrix_t restated on the CPU; pattern as chidg_b200.mesh.BlockPattern."""

    def __init__(self, pat):
        L = lib()
        self.pat = pat
        self._keep = [np.ascontiguousarray(a, dtype=np.int32) for a in
                      (pat.elem_nvars, pat.elem_nterms, pat.elem_proc, pat.blk_row_elem, pat.blk_row_time,
                       pat.blk_col_elem, pat.blk_col_time, pat.blk_kind)]
        k = self._keep
        p = lambda a: a.ctypes.data_as(I32P)
        self.h = L.orc_matrix_create(pat.nelem, pat.ntime, p(k[0]), p(k[1]), p(k[2]), pat.nblocks, p(k[3]), p(k[4]),
                                     p(k[5]), p(k[6]), p(k[7]))
        if not self.h:
            raise ValueError("oracle: invalid pattern")
        self.nval = L.orc_matrix_nvalues(self.h)
        self.n = L.orc_matrix_nvec(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_matrix_destroy(self.h)
            self.h = None

    def set_values(self, vals):
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        assert vals.size == self.nval
        lib().orc_matrix_set_values(self.h, _dp(vals))

    def get_values(self):
        out = np.empty(self.nval)
        lib().orc_matrix_get_values(self.h, _dp(out))
        return out

    def set_transposed(self, transposed: bool = True):
        """chidg_matrix_t%transposed: mv computes A^T x, ILU0 / Jacobi factor A^T."""
        lib().orc_matrix_set_transposed(self.h, int(bool(transposed)))

    def mv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n)
        lib().orc_mv(self.h, _dp(x), _dp(y))
        return y

    def norm(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        return lib().orc_norm(self.h, _dp(x))


class OraclePrecon:
    def __init__(self, A: OracleMatrix, kind):
        if isinstance(kind, str):
            kind = PRECON_NAMES[kind.lower()]
        self.A = A
        self.h = lib().orc_precon_create(A.h, kind)
        if not self.h:
            raise ValueError("oracle: cannot create preconditioner")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_precon_destroy(self.h)
            self.h = None

    def update(self):
        st = lib().orc_precon_update(self.h, self.A.h)
        if st:
            raise ArithmeticError(f"oracle precon update failed ({st}), element {lib().orc_precon_error_elem(self.h)}")

    def apply(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        z = np.empty(self.A.n)
        st = lib().orc_precon_apply(self.h, self.A.h, _dp(v), _dp(z))
        if st:
            raise RuntimeError(f"oracle precon apply failed ({st})")
        return z

    def LD(self):
        out = np.empty(self.A.nval)
        lib().orc_precon_get_LD(self.h, _dp(out))
        return out


def fgmres(A: OracleMatrix, M: OraclePrecon, b, opts: Opts = None, hist_cap=4096):
    """fgmres_t%solve restated; returns (x, result dict)."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty(A.n)
    opts = opts or default_opts()
    res = Result()
    hist = np.zeros(hist_cap)
    st = lib().orc_fgmres_solve(A.h, M.h, _dp(b), _dp(x), C.byref(opts), C.byref(res), _dp(hist), hist_cap)
    if st:
        raise ArithmeticError(f"oracle fgmres failed ({st})")
    return x, {"niter": res.niter, "nrestart": res.nrestart, "residual_norm": res.residual_norm,
               "res_estimate": res.res_estimate, "r0norm_initial": res.r0norm_initial,
               "hist": hist[:res.nhist].copy()}


def inv(a):
    a = np.asfortranarray(a, dtype=np.float64)
    n = a.shape[0]
    out = np.empty_like(a, order="F")
    st = lib().orc_inv(n, a.ctypes.data_as(DP), out.ctypes.data_as(DP))
    if st:
        raise ArithmeticError("inv: Matrix is numerically singular!")
    return out


# ---------------------------------------------------------------------------
# chidg_matrix%to_file (src/containers/type_chidg_matrix.f90:1451-1507) with
# messenger%write_line's formatting (src/tools/messenger.f90:505-640, 695-790)
# ---------------------------------------------------------------------------
def _fortran_fixed(s: str, w: int = 24) -> str:
    return "*" * w if len(s) > w else s.rjust(w)


def fortran_F(v: float, w: int = 24, d: int = 14) -> str:
    """Fw.d: [-]digits.d-digits, right-justified, asterisks when too wide."""
    return _fortran_fixed(f"{v:.{d}f}", w)


def fortran_E(v: float, w: int = 24, d: int = 14) -> str:
    """Ew.d: [-]0.d-digits then E+dd (|exp| <= 99) or +ddd (<= 999)."""
    if v != v:
        return _fortran_fixed("NaN", w)
    if v in (float("inf"), float("-inf")):
        return _fortran_fixed("Infinity" if v > 0 else "-Infinity", w)
    if v == 0.0:
        mant, exp10 = "0" * d, 0
    else:
        m, e = f"{abs(v):.{d - 1}e}".split("e")
        mant, exp10 = m.replace(".", ""), int(e) + 1
    sign = "-" if v < 0 else ""
    ex = f"E{'-' if exp10 < 0 else '+'}{abs(exp10):02d}" if abs(exp10) <= 99 else f"{'-' if exp10 < 0 else '+'}{abs(exp10):03d}"
    return _fortran_fixed(f"{sign}0.{mant}{ex}", w)


def _column(s: str, width: int = 25) -> str:
    s = s.strip()
    while len(s) < width:
        s = " " + s + " "
    return s[:width]


def _real_field(v: float) -> str:
    a = abs(v)
    if a < 0.1:
        s = fortran_E(v)
    elif 0.1 < a < 1.e9:
        s = fortran_F(v)
    else:
        s = fortran_E(v)
    return _column(s)


def to_file_text(pat, vals) -> str:
    """The file chidg_matrix%to_file writes for this pattern and these values:
    per time level, element and LOCAL block (storage order) the entries column
    by column, list-directed (one leading blank), fields joined by ','."""
    voff, _ = pat.value_offsets()
    nr, nc = pat.block_dims()
    out = []
    for t in range(pat.ntime):
        for e in range(pat.nelem):
            ks = [k for k in range(pat.nblocks) if pat.blk_kind[k] == 0 and pat.blk_row_elem[k] == e
                  and pat.blk_row_time[k] == t]
            nblk = _column(str(len(ks)))
            for k in ks:
                b, c = int(nr[k]), int(nc[k])
                r0, c0 = 1 + b * e, 1 + b * int(pat.blk_col_elem[k])
                blk = vals[voff[k]:voff[k] + b * c]
                for j in range(c):
                    for i in range(b):
                        out.append(" " + ",".join([_column(str(r0 + i)), _column(str(c0 + j)), nblk,
                                                    _real_field(float(blk[i + j * b]))]) + "\n")
    return "".join(out)
