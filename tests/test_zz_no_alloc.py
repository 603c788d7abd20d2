"""chidg_gpu_dot_noalloc: the dot product for callers that cannot allocate
device memory when they reduce (inside a stream capture, or under a
framework's own memory pool).  Its partial sums live in a fixed array inside
the library, so the call itself allocates nothing.

Checked through the C ABI against the existing allocating entry point
(chidg_gpu_vector_dot) on the same data, for two calls in a row: the second
call uses a shorter vector and different values, so any partial sums left
behind by the first call would show up.  Collected last (file name) so a
stop-at-first-failure run has run every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh

pytestmark = pytest.mark.gpu

REL_TOL = 1e-13   # the tolerance of the allocating dot in tests/test_gpu_parity.py


def _allocating_dot(x, y):
    """Reference value: chidg_gpu_vector_dot on library vectors with the same data."""
    n = x.size
    pat = mesh.box_pattern(n, 1, 1, 1, 1)     # P0 scalar line: vector length n
    A = api.ChidgMatrix(pat)
    xv, yv = api.ChidgVector(A, x), api.ChidgVector(A, y)
    return api.dot(xv, yv)


def test_dot_noalloc_matches_allocating_dot_twice():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    result = torch.zeros(1, dtype=torch.float64, device=dev)
    for n, seed in ((1_000_003, 1), (70_001, 2)):
        x = mesh.synth_vector(n, seed=seed)
        y = mesh.synth_vector(n, seed=seed + 10)
        xd = torch.from_numpy(x).to(dev)
        yd = torch.from_numpy(y).to(dev)
        st = L.chidg_gpu_dot_noalloc(0, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), n,
                                     C.c_void_p(result.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == _lib.OK
        torch.cuda.synchronize(dev)
        got = float(result.item())
        expect = _allocating_dot(x, y)
        assert got == pytest.approx(expect, rel=REL_TOL)


def test_dot_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda:0")
    buf = torch.zeros(2, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    too_big = 4096 * 16384 + 1
    assert L.chidg_gpu_dot_noalloc(0, p, p, too_big, p, None) == _lib.EINVAL
    assert L.chidg_gpu_dot_noalloc(0, p, p, -1, p, None) == _lib.EINVAL
