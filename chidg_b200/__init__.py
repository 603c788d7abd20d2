"""B200-native implicit linear-solve path for ChiDG.

chidg_matrix_t block-sparse matvec, block-ILU0 and RAS+ILU0 preconditioners
and the restarted FGMRES solver as hand-written sm_100a CUDA kernels behind
the C ABI of include/chidg_gpu.h.  `chidg_b200.api` mirrors the reference's
Fortran interfaces (fgmres_t, precon_ILU0_t, precon_RASILU0_t, chidg_matrix_t,
chidg_vector_t) for Python callers and tests.
"""
from . import _lib  # noqa: F401
from .mesh import box_pattern, nterms_of_order, synth_values, synth_vector  # noqa: F401

__all__ = ["box_pattern", "nterms_of_order", "synth_values", "synth_vector"]
