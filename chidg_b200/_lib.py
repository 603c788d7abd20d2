"""ctypes bindings of the C ABI declared in include/chidg_gpu.h.

The CUDA library (libchidg_gpu.so) is built in-tree by chidg_b200/build.py.
Loading fails loudly when it is missing: there is no CPU fallback for any
entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchidg_gpu.so")
SYNTH_PATH = os.path.join(HERE, "libchidg_synth.so")

OK, EINVAL, ENOMEM, ESINGULAR, ENONFINITE, ETIMEOUT, ENOTCONVERGED, ECUDA, ESTATE = range(9)
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM", 3: "ESINGULAR", 4: "ENONFINITE", 5: "ETIMEOUT",
                6: "ENOTCONVERGED", 7: "ECUDA", 8: "ESTATE"}

BLK_LOCAL, BLK_CHIMERA, BLK_BC, BLK_HB = 0, 1, 2, 3
PRECON_IDENTITY, PRECON_JACOBI, PRECON_ILU0, PRECON_RASILU0, PRECON_HB = 0, 1, 2, 3, 4
FP64, MIXED_FP32, MIXED_BF16, MIXED_PRECON_FP32 = 0, 1, 2, 3
ORTH_CGS, ORTH_MGS = 0, 1
SCHED_LEVELS, SCHED_DATAFLOW, SCHED_TASKS, SCHED_STREAM = 0, 1, 2, 3

I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)
DP = C.POINTER(C.c_double)
VP = C.c_void_p


class EulerBoxDesc(C.Structure):
    """chidg_gpu_euler_box"""
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("order", C.c_int32),
                ("lo", C.c_double * 3), ("hi", C.c_double * 3), ("bc", C.c_int32 * 6),
                ("rho_inf", C.c_double), ("p_inf", C.c_double), ("vel_inf", C.c_double * 3)]


EULER_FARFIELD, EULER_EXTRAPOLATE = 0, 1


class EulerSystemDesc(C.Structure):
    """chidg_gpu_euler_system"""
    _fields_ = [("box", EulerBoxDesc), ("ntime", C.c_int32), ("level_vel", DP), ("D", DP), ("mass", DP),
                ("q0", DP), ("cfl", C.c_double)]


# chidg_gpu_fill_fn
FILL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32)


class Pattern(C.Structure):
    _fields_ = [("nelem", C.c_int32), ("ntime", C.c_int32), ("elem_nvars", I32P), ("elem_nterms", I32P),
                ("elem_proc", I32P), ("nblocks", C.c_int64), ("blk_row_elem", I32P), ("blk_row_time", I32P),
                ("blk_col_elem", I32P), ("blk_col_time", I32P), ("blk_kind", I32P)]


class FgmresOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("rtol", C.c_double), ("nmax", C.c_int32), ("nkrylov", C.c_int32),
                ("orthogonalization", C.c_int32), ("inner_fgmres", C.c_int32), ("inner_tol", C.c_double),
                ("inner_rtol", C.c_double), ("inner_nmax", C.c_int32), ("inner_nkrylov", C.c_int32),
                ("inner_orthogonalization", C.c_int32), ("use_controller", C.c_int32), ("precision", C.c_int32),
                ("mixed_inner_nkrylov", C.c_int32), ("mixed_inner_rtol", C.c_double),
                ("mixed_inner_nmax", C.c_int32)]


class FgmresResult(C.Structure):
    _fields_ = [("niter", C.c_int32), ("nrestart", C.c_int32), ("inner_iters", C.c_int32), ("nhist", C.c_int32),
                ("residual_norm", C.c_double), ("res_estimate", C.c_double), ("r0norm_initial", C.c_double),
                ("seconds", C.c_double)]


# name -> (restype, argtypes)
PROTOTYPES = {
    "chidg_gpu_ctx_create": (C.c_int, [C.c_int, VP, C.POINTER(VP)]),
    "chidg_gpu_ctx_destroy": (C.c_int, [VP]),
    "chidg_gpu_ctx_sync": (C.c_int, [VP]),
    "chidg_gpu_last_error": (C.c_int, [VP, C.c_char_p, C.c_int32]),
    "chidg_gpu_error_element": (C.c_int, [VP, I32P]),
    "chidg_gpu_launch_count": (C.c_int, [VP, I64P]),
    "chidg_gpu_ctx_set_profiling": (C.c_int, [VP, C.c_int32]),
    "chidg_gpu_ctx_kernel_time": (C.c_int, [VP, C.c_int32, DP, I64P]),
    "chidg_gpu_host_alloc": (C.c_int, [C.c_size_t, C.POINTER(VP)]),
    "chidg_gpu_host_free": (C.c_int, [VP]),
    "chidg_gpu_matrix_create": (C.c_int, [VP, C.POINTER(Pattern), C.POINTER(VP)]),
    "chidg_gpu_matrix_destroy": (C.c_int, [VP]),
    "chidg_gpu_matrix_nvalues": (C.c_int, [VP, I64P]),
    "chidg_gpu_matrix_nvec": (C.c_int, [VP, I64P]),
    "chidg_gpu_matrix_upload": (C.c_int, [VP, VP]),
    "chidg_gpu_matrix_upload_range": (C.c_int, [VP, VP, C.c_int64, C.c_int64]),
    "chidg_gpu_matrix_upload_blocks": (C.c_int, [VP, C.POINTER(VP)]),
    "chidg_gpu_matrix_upload_device": (C.c_int, [VP, VP]),
    "chidg_gpu_matrix_download": (C.c_int, [VP, VP]),
    "chidg_gpu_matrix_clear": (C.c_int, [VP]),
    "chidg_gpu_matrix_scale_diagonal": (C.c_int, [VP, DP, DP]),
    "chidg_gpu_matrix_stamp": (C.c_int, [VP, I64P]),
    "chidg_gpu_matrix_set_transposed": (C.c_int, [VP, C.c_int32]),
    "chidg_gpu_matrix_get_transposed": (C.c_int, [VP, C.POINTER(C.c_int32)]),
    "chidg_gpu_matrix_to_file": (C.c_int, [VP, C.c_char_p]),
    "chidg_gpu_matrix_save": (C.c_int, [VP, C.c_char_p]),
    "chidg_gpu_matrix_load": (C.c_int, [VP, C.c_char_p, C.POINTER(VP)]),
    "chidg_gpu_matrix_get_pattern": (C.c_int, [VP, C.POINTER(C.c_int32), C.POINTER(C.c_int32), I64P, I32P, I32P, I32P,
                                               I32P, I32P, I32P, I32P, I32P]),
    "chidg_gpu_vector_create": (C.c_int, [VP, C.POINTER(VP)]),
    "chidg_gpu_vector_destroy": (C.c_int, [VP]),
    "chidg_gpu_vector_upload": (C.c_int, [VP, VP]),
    "chidg_gpu_vector_upload_range": (C.c_int, [VP, VP, C.c_int64, C.c_int64]),
    "chidg_gpu_vector_download": (C.c_int, [VP, VP]),
    "chidg_gpu_vector_upload_device": (C.c_int, [VP, VP]),
    "chidg_gpu_vector_device_ptr": (C.c_int, [VP, C.POINTER(VP)]),
    "chidg_gpu_vector_clear": (C.c_int, [VP]),
    "chidg_gpu_vector_copy": (C.c_int, [VP, VP]),
    "chidg_gpu_vector_axpy": (C.c_int, [VP, C.c_double, VP]),
    "chidg_gpu_vector_scale": (C.c_int, [VP, C.c_double]),
    "chidg_gpu_vector_dot": (C.c_int, [VP, VP, DP]),
    "chidg_gpu_vector_norm": (C.c_int, [VP, DP]),
    "chidg_gpu_dot_noalloc": (C.c_int, [C.c_int, VP, VP, C.c_int64, VP, VP]),
    "chidg_gpu_matvec": (C.c_int, [VP, VP, VP]),
    "chidg_gpu_vector_norm_fields": (C.c_int, [VP, VP, C.c_int32]),
    "chidg_gpu_selftest_bounded_waits": (C.c_int, [VP, C.c_int64, C.POINTER(C.c_int32)]),
    "chidg_gpu_autotune": (C.c_int, [VP, VP, C.c_int32, C.c_int32]),
    "chidg_gpu_euler_assemble_at": (C.c_int, [VP, VP, C.c_int32, VP, VP, C.c_int32]),
    "chidg_gpu_euler_pseudo_timestep_at": (C.c_int, [VP, VP, C.c_int32, VP, DP, DP]),
    "chidg_gpu_euler_assemble_level": (C.c_int, [VP, VP, C.c_int32, VP, VP, C.c_int32]),
    "chidg_gpu_euler_pseudo_timestep_level": (C.c_int, [VP, VP, C.c_int32, VP, DP, DP]),
    "chidg_gpu_hb_coupling": (C.c_int, [VP, C.c_int32, DP, DP, VP, VP, C.c_int32]),
    "chidg_gpu_euler_assemble_level_at": (C.c_int, [VP, VP, C.c_int32, C.c_int32, VP, VP, C.c_int32]),
    "chidg_gpu_hb_coupling_at": (C.c_int, [VP, C.c_int32, C.c_int32, C.c_int32, DP, DP, VP, VP, C.c_int32]),
    "chidg_gpu_euler_pseudo_transient_at": (C.c_int, [VP, VP, C.c_int32, VP, VP, DP, DP]),
    "chidg_gpu_euler_fill_system": (C.c_int, [VP, VP, VP, VP, VP, C.c_int32]),
    "chidg_gpu_vector_mass_scale": (C.c_int, [VP, VP, DP, DP]),
    "chidg_gpu_stream_shape_get": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, I32P, I32P, I32P]),
    "chidg_gpu_stream_shape_set": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "chidg_gpu_euler_create": (C.c_int, [VP, VP, C.POINTER(VP)]),
    "chidg_gpu_euler_destroy": (C.c_int, [VP]),
    "chidg_gpu_euler_assemble": (C.c_int, [VP, VP, VP, VP]),
    "chidg_gpu_euler_pseudo_timestep": (C.c_int, [VP, VP, DP, DP]),
    "chidg_gpu_serve_create": (C.c_int, [C.c_int, C.c_int32, C.c_int64, C.c_int32, C.c_int32, VP, C.POINTER(VP)]),
    "chidg_gpu_serve_submit": (C.c_int, [VP, VP, VP, VP, C.POINTER(C.c_int64)]),
    "chidg_gpu_serve_wait": (C.c_int, [VP, C.c_int64, VP, VP, VP]),
    "chidg_gpu_serve_stats": (C.c_int, [VP, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "chidg_gpu_serve_destroy": (C.c_int, [VP]),
    "chidg_gpu_serve_submit_fill": (C.c_int, [VP, VP, VP, VP, C.POINTER(C.c_int64)]),
    "chidg_gpu_serve_batch_log": (C.c_int, [VP, C.c_int64, DP]),
    "chidg_gpu_precon_create": (C.c_int, [VP, C.c_int32, C.POINTER(VP)]),
    "chidg_gpu_precon_destroy": (C.c_int, [VP]),
    "chidg_gpu_precon_update": (C.c_int, [VP, VP, C.c_int32]),
    "chidg_gpu_precon_apply": (C.c_int, [VP, VP, VP, VP]),
    "chidg_gpu_precon_download_LD": (C.c_int, [VP, VP]),
    "chidg_gpu_precon_download_LD32": (C.c_int, [VP, VP]),
    "chidg_gpu_precon_stamp": (C.c_int, [VP, I64P]),
    "chidg_gpu_precon_set_schedule": (C.c_int, [VP, C.c_int32]),
    "chidg_gpu_fgmres_solve": (C.c_int, [VP, VP, VP, VP, C.POINTER(FgmresOpts), C.POINTER(FgmresResult), DP,
                                         C.c_int32]),
    "chidg_gpu_fgmres_default_opts": (C.c_int, [C.POINTER(FgmresOpts)]),
    "chidg_gpu_fgmres_solve_batched": (C.c_int, [VP, VP, C.c_int32, I32P, VP, VP, C.POINTER(FgmresOpts),
                                                 C.POINTER(FgmresResult), DP, C.c_int32]),
}

_lib = None
_synth = None


class ChidgGpuError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")


def lib():
    """Load libchidg_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m chidg_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def synth():
    """Load the host-only synthetic input generator."""
    global _synth
    if _synth is None:
        if not os.path.exists(SYNTH_PATH):
            raise ImportError(f"{SYNTH_PATH} is missing: run `python -m chidg_b200.build`")
        S = C.CDLL(SYNTH_PATH)
        S.chidg_synth_blocks.restype = C.c_int
        S.chidg_synth_blocks.argtypes = [C.c_int64, I32P, I32P, I64P, I32P, C.c_uint64, DP, DP, C.c_int]
        S.chidg_synth_vector.restype = C.c_int
        S.chidg_synth_vector.argtypes = [C.c_int64, C.c_uint64, DP, C.c_int]
        _synth = S
    return _synth
