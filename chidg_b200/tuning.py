"""The project autotuner of the streamed kernels' launch shapes.

`autotune(A, M, precision)` measures, on the device, every candidate shape
(consumer warps, ring stages, bytes per stage) of the four streamed kernel
kinds that an FGMRES solve with M and A launches -- forward sweep, backward
sweep, backward sweep with the matvec rows, matvec -- and keeps the fastest of
each for A's block-size class and value width (chidg_gpu_autotune).  With a
cache file, shapes already measured for that (kind, class, width) are loaded
instead of measured again, and new measurements are added to the file (JSON).
"""
from __future__ import annotations

import ctypes as C
import json
import os

from . import _lib

KINDS = {0: "forward", 1: "backward", 2: "backward_matvec", 3: "matvec"}
PRECISION_WIDTH = {"fp64": (8, 8), "mixed_precon_fp32": (4, 8), "mixed_fp32": (4, 4), "mixed_bf16": (2, 2)}
CLASSES = (64, 160, 384, 1024)


def size_class(max_b: int) -> int:
    for c in CLASSES:
        if max_b <= c:
            return c
    raise ValueError("blocks over 1024 rows have no streamed shape")


def get_shape(kind: int, max_b: int, value_bytes: int) -> dict:
    w, s, b = C.c_int32(), C.c_int32(), C.c_int32()
    st = _lib.lib().chidg_gpu_stream_shape_get(kind, max_b, value_bytes, C.byref(w), C.byref(s), C.byref(b))
    if st:
        raise ValueError(f"stream_shape_get failed ({st})")
    return {"warps": w.value, "stages": s.value, "stage_bytes": b.value}


def set_shape(kind: int, max_b: int, value_bytes: int, shape: dict) -> None:
    st = _lib.lib().chidg_gpu_stream_shape_set(kind, max_b, value_bytes, int(shape["warps"]), int(shape["stages"]),
                                               int(shape["stage_bytes"]))
    if st:
        raise ValueError(f"stream_shape_set refused {shape} ({st})")


def _key(kind: int, max_b: int, value_bytes: int) -> str:
    return f"{KINDS[kind]}/b<={size_class(max_b)}/{value_bytes}B"


def autotune(A, M, precision: str = "fp64", reps: int = 3, cache: str | None = None) -> dict:
    """Shapes for A's block-size class in `precision`; M must be updated for A in
    that precision.  Returns {key: shape}; `cache` (a JSON file) is read first
    and updated after a measurement."""
    from .api import PRECISIONS
    max_b = int(A.pattern.bsize().max())
    wb, wm = PRECISION_WIDTH[precision]
    widths = {0: wb, 1: wb, 2: wb, 3: wm}
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as f:
            table = json.load(f)
    keys = {k: _key(k, max_b, widths[k]) for k in KINDS}
    if all(keys[k] in table for k in KINDS):
        for k in KINDS:
            set_shape(k, max_b, widths[k], table[keys[k]])
    else:
        A.ctx.check(_lib.lib().chidg_gpu_autotune(M.h, A.h, PRECISIONS[precision], int(reps)), "autotune")
        for k in KINDS:
            table[keys[k]] = get_shape(k, max_b, widths[k])
        if cache:
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
    return {keys[k]: table[keys[k]] for k in KINDS}
