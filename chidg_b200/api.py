"""Python mirror of the reference's linear-solve interfaces, backed by the
CUDA library through the C ABI (include/chidg_gpu.h).

Reference interface -> class here
  chidg_matrix_t   (src/containers/type_chidg_matrix.f90)        ChidgMatrix
  chidg_vector_t   (src/containers/type_chidg_vector.f90)        ChidgVector
  chidg_mv         (src/containers/operator_chidg_mv.f90:46)     chidg_mv
  dot              (src/containers/operator_chidg_dot.f90:30)    dot
  preconditioner_t (src/preconditioners/type_preconditioner.f90) Preconditioner
  create_preconditioner (src/preconditioners/mod_preconditioner.f90:49)
  fgmres_t         (src/linear_solvers/type_fgmres.f90)          FGMRES
  create_linear_solver  (src/linear_solvers/mod_linear_solver.f90:27)

Errors: a nonzero status raises ChidgGpuError, the counterpart of the
reference's chidg_signal(FATAL, ...).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib, mesh
from ._lib import ChidgGpuError

_ctx_default = {}


class Context:
    """One CUDA device + one stream (optionally the caller's, e.g. a torch stream)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.L = _lib.lib()
        h = C.c_void_p()
        st = self.L.chidg_gpu_ctx_create(int(device), C.c_void_p(stream) if stream else None, C.byref(h))
        if st:
            raise ChidgGpuError(st, f"cannot create a context on device {device}")
        self.h = h
        self.device = device

    def check(self, st, what=""):
        if st:
            buf = C.create_string_buffer(512)
            self.L.chidg_gpu_last_error(self.h, buf, 512)
            el = C.c_int32(-1)
            self.L.chidg_gpu_error_element(self.h, C.byref(el))
            msg = f"{what}: {buf.value.decode(errors='replace')}"
            err = ChidgGpuError(st, msg)
            err.element = el.value
            raise err

    def sync(self):
        self.check(self.L.chidg_gpu_ctx_sync(self.h), "sync")

    def launches(self) -> int:
        c = C.c_int64(0)
        self.check(self.L.chidg_gpu_launch_count(self.h, C.byref(c)), "launch_count")
        return c.value

    PROFILE_CLASSES = {"matvec": 0, "ilu_forward": 1, "ilu_backward": 2, "factor": 3, "matvec_fp32": 4,
                       "ilu_lowp": 5, "factor_gemm": 6, "factor_inverse": 7, "ilu_backward_matvec": 8}

    def set_profiling(self, on: bool):
        self.check(self.L.chidg_gpu_ctx_set_profiling(self.h, int(bool(on))), "set_profiling")

    def kernel_times(self) -> dict:
        """{class: (total_ms, count)} of the event-timed kernel classes."""
        out = {}
        for name, c in self.PROFILE_CLASSES.items():
            ms, n = C.c_double(), C.c_int64()
            self.check(self.L.chidg_gpu_ctx_kernel_time(self.h, c, C.byref(ms), C.byref(n)), "kernel_time")
            out[name] = (ms.value, n.value)
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.chidg_gpu_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_context(device: int = 0) -> Context:
    if device not in _ctx_default:
        _ctx_default[device] = Context(device)
    return _ctx_default[device]


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class ChidgMatrix:
    """chidg_matrix_t with backend='cuda': block pattern + FP64 block values on the GPU."""

    def __init__(self, pattern, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.pattern = pattern
        self._pat = pattern.as_struct()
        h = C.c_void_p()
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_create(self.ctx.h, C.byref(self._pat), C.byref(h)), "matrix_create")
        self.h = h
        n = C.c_int64()
        self.ctx.L.chidg_gpu_matrix_nvalues(self.h, C.byref(n))
        self.nvalues = n.value
        self.ctx.L.chidg_gpu_matrix_nvec(self.h, C.byref(n))
        self.n = n.value

    def upload(self, values: np.ndarray):
        values = np.ascontiguousarray(values, dtype=np.float64)
        if values.size != self.nvalues:
            raise ValueError(f"expected {self.nvalues} values, got {values.size}")
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_upload(self.h, _ptr(values)), "matrix_upload")
        self.ctx.sync()

    def upload_parts(self, parts):
        """Consecutive pieces of the packed values (e.g. one per system of a
        batch), uploaded in place without first joining them on the host."""
        parts = [np.ascontiguousarray(p, dtype=np.float64) for p in parts]
        if sum(p.size for p in parts) != self.nvalues:
            raise ValueError(f"expected {self.nvalues} values in total")
        first = 0
        for p in parts:
            self.upload_range(p, first)
            first += p.size
        self.ctx.sync()

    def upload_range(self, values: np.ndarray, first: int):
        """values into the packed entries first.. (queued on the context's
        stream: from page-locked memory the array must live until a sync)."""
        if values.dtype != np.float64 or not values.flags.c_contiguous:
            raise ValueError("upload_range: a contiguous float64 array")
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_upload_range(self.h, _ptr(values), int(first), values.size),
                       "matrix_upload_range")

    def upload_blocks(self, blocks):
        """One array per block (each densematrix_t%mat), in pattern order."""
        arrs = [np.asfortranarray(b, dtype=np.float64) for b in blocks]
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_upload_blocks(self.h, ptrs), "matrix_upload_blocks")
        self.ctx.sync()

    def upload_device(self, dev_ptr: int):
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_upload_device(self.h, C.c_void_p(dev_ptr)), "matrix_upload_device")

    def download(self) -> np.ndarray:
        out = np.empty(self.nvalues)
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_download(self.h, _ptr(out)), "matrix_download")
        return out

    def clear(self):
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_clear(self.h), "matrix_clear")

    def scale_diagonal(self, mass: np.ndarray, scale: np.ndarray):
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        scale = np.ascontiguousarray(scale, dtype=np.float64)
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_scale_diagonal(self.h, mass.ctypes.data_as(_lib.DP),
                                                                  scale.ctypes.data_as(_lib.DP)), "scale_diagonal")

    @property
    def stamp(self) -> int:
        s = C.c_int64()
        self.ctx.L.chidg_gpu_matrix_stamp(self.h, C.byref(s))
        return s.value

    @property
    def transposed(self) -> bool:
        """chidg_matrix_t%transposed: products, ILU0 and Jacobi act on A^T."""
        t = C.c_int32()
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_get_transposed(self.h, C.byref(t)), "get_transposed")
        return bool(t.value)

    @transposed.setter
    def transposed(self, value: bool):
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_set_transposed(self.h, int(bool(value))), "set_transposed")

    def to_file(self, path: str):
        """chidg_matrix%to_file: the LOCAL blocks as ChiDG's text listing."""
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_to_file(self.h, os.fsencode(path)), "to_file")

    def save(self, path: str):
        """Binary image (pattern, transposed flag, values) for ChidgMatrix.load."""
        self.ctx.check(self.ctx.L.chidg_gpu_matrix_save(self.h, os.fsencode(path)), "save")

    @classmethod
    def load(cls, path: str, ctx: Context | None = None) -> "ChidgMatrix":
        ctx = ctx or default_context()
        h = C.c_void_p()
        ctx.check(ctx.L.chidg_gpu_matrix_load(ctx.h, os.fsencode(path), C.byref(h)), "load")
        self = cls.__new__(cls)
        self.ctx, self.h = ctx, h
        ne, nt, nb = C.c_int32(), C.c_int32(), C.c_int64()
        ctx.check(ctx.L.chidg_gpu_matrix_get_pattern(h, C.byref(ne), C.byref(nt), C.byref(nb), *([None] * 8)), "get_pattern")
        el = [np.empty(ne.value, dtype=np.int32) for _ in range(3)]
        bl = [np.empty(nb.value, dtype=np.int32) for _ in range(5)]
        ctx.check(ctx.L.chidg_gpu_matrix_get_pattern(h, None, None, None, *[a.ctypes.data_as(_lib.I32P) for a in el + bl]),
                  "get_pattern")
        diag = (bl[0] == bl[2]) & (bl[1] == bl[3]) & (bl[4] == _lib.BLK_LOCAL)
        self.pattern = mesh.BlockPattern(nelem=ne.value, ntime=nt.value, elem_nvars=el[0], elem_nterms=el[1],
                                         elem_proc=el[2], blk_row_elem=bl[0], blk_row_time=bl[1], blk_col_elem=bl[2],
                                         blk_col_time=bl[3], blk_kind=bl[4],
                                         blk_face=np.where(diag, mesh.DIAG, mesh.OTHER).astype(np.int32))
        self._pat = self.pattern.as_struct()
        n = C.c_int64()
        ctx.L.chidg_gpu_matrix_nvalues(h, C.byref(n))
        self.nvalues = n.value
        ctx.L.chidg_gpu_matrix_nvec(h, C.byref(n))
        self.n = n.value
        return self

    def release(self):
        if getattr(self, "h", None):
            self.ctx.L.chidg_gpu_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class ChidgVector:
    """chidg_vector_t with backend='cuda'."""

    def __init__(self, A: ChidgMatrix, values: np.ndarray | None = None):
        self.A = A
        self.ctx = A.ctx
        h = C.c_void_p()
        self.ctx.check(self.ctx.L.chidg_gpu_vector_create(A.h, C.byref(h)), "vector_create")
        self.h = h
        self.n = A.n
        if values is not None:
            self.upload(values)

    def upload(self, values):
        values = np.ascontiguousarray(values, dtype=np.float64)
        if values.size != self.n:
            raise ValueError("vector size mismatch")
        self.ctx.check(self.ctx.L.chidg_gpu_vector_upload(self.h, _ptr(values)), "vector_upload")
        self.ctx.sync()

    def upload_parts(self, parts):
        """Consecutive pieces of the vector, uploaded in place."""
        parts = [np.ascontiguousarray(p, dtype=np.float64) for p in parts]
        if sum(p.size for p in parts) != self.n:
            raise ValueError("vector size mismatch")
        first = 0
        for p in parts:
            self.upload_range(p, first)
            first += p.size
        self.ctx.sync()

    def upload_range(self, values: np.ndarray, first: int):
        """values into entries first.. (queued, as ChidgMatrix.upload_range)."""
        if values.dtype != np.float64 or not values.flags.c_contiguous:
            raise ValueError("upload_range: a contiguous float64 array")
        self.ctx.check(self.ctx.L.chidg_gpu_vector_upload_range(self.h, _ptr(values), int(first), values.size),
                       "vector_upload_range")

    def download(self) -> np.ndarray:
        out = np.empty(self.n)
        self.ctx.check(self.ctx.L.chidg_gpu_vector_download(self.h, _ptr(out)), "vector_download")
        return out

    def device_ptr(self) -> int:
        p = C.c_void_p()
        self.ctx.L.chidg_gpu_vector_device_ptr(self.h, C.byref(p))
        return p.value

    def clear(self):
        self.ctx.check(self.ctx.L.chidg_gpu_vector_clear(self.h), "vector_clear")

    def assign_mass_scaled(self, x: "ChidgVector", mass: np.ndarray, scale: np.ndarray):
        """self = scale[e, f] mass_e x on every element, time level and field
        segment (pseudo_transient_scaling); mass and scale packed as
        ChidgMatrix.scale_diagonal takes them."""
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        scale = np.ascontiguousarray(scale, dtype=np.float64)
        self.ctx.check(self.ctx.L.chidg_gpu_vector_mass_scale(x.h, self.h, mass.ctypes.data_as(_lib.DP),
                                                              scale.ctypes.data_as(_lib.DP)), "vector_mass_scale")

    def copy_from(self, other: "ChidgVector"):
        self.ctx.check(self.ctx.L.chidg_gpu_vector_copy(self.h, other.h), "vector_copy")

    def axpy(self, a: float, x: "ChidgVector"):
        self.ctx.check(self.ctx.L.chidg_gpu_vector_axpy(self.h, float(a), x.h), "vector_axpy")

    def scale(self, a: float):
        self.ctx.check(self.ctx.L.chidg_gpu_vector_scale(self.h, float(a)), "vector_scale")

    def norm(self) -> float:
        out = C.c_double()
        self.ctx.check(self.ctx.L.chidg_gpu_vector_norm(self.h, C.byref(out)), "vector_norm")
        return out.value

    def norm_fields(self, nfields: int | None = None) -> np.ndarray:
        """chidg_vector%norm_fields: the L2 norm of each field over all elements,
        time levels and modes (every element with the same field count)."""
        nf = int(self.A.pattern.elem_nvars[0]) if nfields is None else int(nfields)
        out = np.empty(nf)
        self.ctx.check(self.ctx.L.chidg_gpu_vector_norm_fields(self.h, _ptr(out), nf), "vector_norm_fields")
        return out

    # chidg_vector_t's overloaded operators (type_chidg_vector.f90:1740-2084):
    # each returns a new vector
    def _new_copy(self) -> "ChidgVector":
        out = ChidgVector(self.A)
        out.copy_from(self)
        return out

    def __add__(self, other: "ChidgVector") -> "ChidgVector":
        out = self._new_copy()
        out.axpy(1.0, other)
        return out

    def __sub__(self, other: "ChidgVector") -> "ChidgVector":
        out = self._new_copy()
        out.axpy(-1.0, other)
        return out

    def __neg__(self) -> "ChidgVector":
        out = self._new_copy()
        out.scale(-1.0)
        return out

    def __mul__(self, a: float) -> "ChidgVector":
        out = self._new_copy()
        out.scale(float(a))
        return out

    __rmul__ = __mul__

    def __truediv__(self, a: float) -> "ChidgVector":
        out = self._new_copy()
        out.scale(1.0 / float(a))
        return out

    def release(self):
        if getattr(self, "h", None):
            self.ctx.L.chidg_gpu_vector_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def dot(x: ChidgVector, y: ChidgVector) -> float:
    out = C.c_double()
    x.ctx.check(x.ctx.L.chidg_gpu_vector_dot(x.h, y.h, C.byref(out)), "dot")
    return out.value


def chidg_mv(A: ChidgMatrix, x: ChidgVector, y: ChidgVector | None = None) -> ChidgVector:
    y = y or ChidgVector(A)
    A.ctx.check(A.ctx.L.chidg_gpu_matvec(A.h, x.h, y.h), "chidg_mv")
    return y


PRECON_KINDS = {"identity": _lib.PRECON_IDENTITY, "jacobi": _lib.PRECON_JACOBI, "ilu0": _lib.PRECON_ILU0,
                "rasilu0": _lib.PRECON_RASILU0, "hb": _lib.PRECON_HB}
PRECISIONS = {"fp64": _lib.FP64, "mixed_fp32": _lib.MIXED_FP32, "mixed_bf16": _lib.MIXED_BF16,
              "mixed_precon_fp32": _lib.MIXED_PRECON_FP32}


class Preconditioner:
    """preconditioner_t: init / update / apply / tear_down."""

    def __init__(self, kind: str, schedule: str = "stream"):
        self.kind = kind.lower()
        self.schedule = schedule
        if self.kind not in PRECON_KINDS:
            raise ValueError(f"create_preconditioner: invalid preconditioner '{kind}'")
        self.h = None
        self.A = None

    def init(self, A: ChidgMatrix):
        self.tear_down()
        self.A = A
        h = C.c_void_p()
        A.ctx.check(A.ctx.L.chidg_gpu_precon_create(A.h, PRECON_KINDS[self.kind], C.byref(h)), f"{self.kind}%init")
        self.h = h
        self.set_schedule(self.schedule)
        return self

    def set_schedule(self, schedule: str):
        """'levels' (one launch per wavefront), 'dataflow' (one launch per sweep,
        row granularity), 'tasks' (one launch per sweep, block granularity) or
        'stream' (the tasks with blocks prefetched into shared memory)."""
        self.schedule = schedule
        if self.h is not None:
            code = {"levels": _lib.SCHED_LEVELS, "dataflow": _lib.SCHED_DATAFLOW, "tasks": _lib.SCHED_TASKS,
                    "stream": _lib.SCHED_STREAM}[schedule]
            self.A.ctx.check(self.A.ctx.L.chidg_gpu_precon_set_schedule(self.h, code), "set_schedule")

    def update(self, A: ChidgMatrix, b=None, precision: str = "fp64"):
        if self.h is None or A is not self.A:
            self.init(A)
        A.ctx.check(A.ctx.L.chidg_gpu_precon_update(self.h, A.h, PRECISIONS[precision]), f"{self.kind}%update")

    def apply(self, A: ChidgMatrix, v: ChidgVector, z: ChidgVector | None = None) -> ChidgVector:
        z = z or ChidgVector(A)
        A.ctx.check(A.ctx.L.chidg_gpu_precon_apply(self.h, A.h, v.h, z.h), f"{self.kind}%apply")
        return z

    def LD(self) -> np.ndarray:
        out = np.empty(self.A.nvalues)
        self.A.ctx.check(self.A.ctx.L.chidg_gpu_precon_download_LD(self.h, _ptr(out)), "LD")
        return out

    def LD32(self) -> np.ndarray:
        """The FP32 factors of the last mixed-precision update."""
        out = np.empty(self.A.nvalues, dtype=np.float32)
        self.A.ctx.check(self.A.ctx.L.chidg_gpu_precon_download_LD32(self.h, _ptr(out)), "LD32")
        return out

    @property
    def stamp(self) -> int:
        s = C.c_int64()
        self.A.ctx.L.chidg_gpu_precon_stamp(self.h, C.byref(s))
        return s.value

    def tear_down(self):
        if self.h is not None and self.A is not None:
            self.A.ctx.L.chidg_gpu_precon_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.tear_down()
        except Exception:
            pass


def create_preconditioner(name: str, schedule: str = "stream") -> Preconditioner:
    return Preconditioner(name, schedule)


class FGMRES:
    """fgmres_t: options with the defaults of linear_solver_t, solve(A, x, b, M)."""

    def __init__(self, **options):
        o = _lib.FgmresOpts()
        _lib.lib().chidg_gpu_fgmres_default_opts(C.byref(o))
        self._o = o
        self.niter = 0
        self.nrestart = 0
        self.inner_iters = 0
        self.residual_norm = 0.0
        self.res_estimate = 0.0
        self.r0norm_initial = 0.0
        self.seconds = 0.0
        self.hist = np.zeros(0)
        self.set(**options)

    def set(self, **options):
        """linear_solver%set (type_linear_solver.f90:113-131)."""
        for k, v in options.items():
            if k in ("orthogonalization", "inner_orthogonalization") and isinstance(v, str):
                v = _lib.ORTH_CGS if v.upper() == "CGS" else _lib.ORTH_MGS
            if k == "precision" and isinstance(v, str):
                v = PRECISIONS[v]
            if k in ("inner_fgmres", "use_controller"):
                v = int(bool(v))
            if not hasattr(self._o, k):
                raise KeyError(k)
            setattr(self._o, k, v)

    def __getattr__(self, k):
        o = self.__dict__.get("_o")
        if o is not None and k in dict(_lib.FgmresOpts._fields_):
            return getattr(o, k)
        raise AttributeError(k)

    def solve(self, A: ChidgMatrix, x: ChidgVector, b: ChidgVector, M: Preconditioner, hist_cap: int = 8192):
        if M.h is None or M.A is not A:
            M.init(A)
        res = _lib.FgmresResult()
        hist = np.zeros(hist_cap)
        st = A.ctx.L.chidg_gpu_fgmres_solve(A.h, M.h, b.h, x.h, C.byref(self._o), C.byref(res),
                                            hist.ctypes.data_as(_lib.DP), hist_cap)
        self.niter, self.nrestart, self.inner_iters = res.niter, res.nrestart, res.inner_iters
        self.residual_norm, self.res_estimate = res.residual_norm, res.res_estimate
        self.r0norm_initial, self.seconds = res.r0norm_initial, res.seconds
        self.hist = hist[:res.nhist].copy()
        A.ctx.check(st, "fgmres%solve")
        return x


    def solve_batched(self, A: ChidgMatrix, x: ChidgVector, b: ChidgVector, M: Preconditioner, sys_elem,
                      hist_cap: int = 1024):
        """Independent systems packed block-diagonally in A (system s owns elements
        sys_elem[s]:sys_elem[s+1]); returns one result dict per system."""
        if M.h is None or M.A is not A:
            M.init(A)
        se = np.ascontiguousarray(sys_elem, dtype=np.int32)
        ns = se.size - 1
        res = (_lib.FgmresResult * ns)()
        hist = np.zeros(ns * hist_cap)
        st = A.ctx.L.chidg_gpu_fgmres_solve_batched(A.h, M.h, ns, se.ctypes.data_as(_lib.I32P), b.h, x.h,
                                                    C.byref(self._o), res, hist.ctypes.data_as(_lib.DP), hist_cap)
        A.ctx.check(st, "fgmres%solve (batched)")
        out = []
        for s in range(ns):
            r = res[s]
            out.append({"niter": r.niter, "nrestart": r.nrestart, "inner_iters": r.inner_iters,
                        "residual_norm": r.residual_norm, "res_estimate": r.res_estimate,
                        "r0norm_initial": r.r0norm_initial, "seconds": r.seconds,
                        "hist": hist[s * hist_cap:s * hist_cap + r.nhist].copy()})
        return out


def create_linear_solver(name: str, **options) -> FGMRES:
    if name.lower() != "fgmres":
        raise ValueError(f"create_linear_solver: invalid linear solver '{name}'")
    return FGMRES(**options)
