"""chidg_gpu_dot_noalloc: the dot product for callers that cannot allocate
device memory when they reduce (a framework that owns all device memory
through its own pool, or a loop that cannot afford the device-wide
synchronisation an allocation may bring).  Its partial sums live in a fixed
array inside the library, so the call itself allocates nothing.

Checked through the C ABI against the existing allocating entry point
(chidg_gpu_vector_dot) on the same data, for calls in a row: a long vector,
then a shorter one, then a longer one again, so partial sums left behind by
an earlier call would be read if a call did not overwrite every partial it
reads.  Collected last (file name) so a stop-at-first-failure run has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh

pytestmark = pytest.mark.gpu

REL_TOL = 1e-13   # the tolerance of the allocating dot in tests/test_gpu_parity.py
MAX_N = 4096 * 16384


def _allocating_dot(x, y):
    """Reference value: chidg_gpu_vector_dot on library vectors with the same data."""
    n = x.size
    pat = mesh.box_pattern(n, 1, 1, 1, 1)     # P0 scalar line: vector length n
    A = api.ChidgMatrix(pat)
    xv, yv = api.ChidgVector(A, x), api.ChidgVector(A, y)
    return api.dot(xv, yv)


def _noalloc_dot(L, xd, yd, n, result, stream):
    import torch
    st = L.chidg_gpu_dot_noalloc(0, C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), n,
                                 C.c_void_p(result.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert st == _lib.OK
    torch.cuda.synchronize(result.device)
    return float(result.item())


def test_dot_noalloc_matches_allocating_dot_in_a_row():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    result = torch.zeros(1, dtype=torch.float64, device=dev)
    for n, seed in ((1_000_003, 1), (70_001, 2), (1_000_003, 3)):
        x = mesh.synth_vector(n, seed=seed)
        y = mesh.synth_vector(n, seed=seed + 10)
        xd = torch.from_numpy(x).to(dev)
        yd = torch.from_numpy(y).to(dev)
        got = _noalloc_dot(L, xd, yd, n, result, stream)
        assert got == pytest.approx(_allocating_dot(x, y), rel=REL_TOL)


def test_dot_noalloc_empty_and_largest_sizes():
    """n = 0 runs only the finishing kernel and must write 0; the largest
    accepted n fills every slot of the scratch array (positive values, so the
    float64 host sum is a tight reference)."""
    import torch
    L = _lib.lib()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    result = torch.full((1,), 7.0, dtype=torch.float64, device=dev)
    buf = torch.zeros(1, dtype=torch.float64, device=dev)
    assert _noalloc_dot(L, buf, buf, 0, result, stream) == 0.0
    g = torch.Generator(device=dev).manual_seed(5)
    x = torch.rand(MAX_N, dtype=torch.float64, device=dev, generator=g)
    y = torch.rand(MAX_N, dtype=torch.float64, device=dev, generator=g)
    got = _noalloc_dot(L, x, y, MAX_N, result, stream)
    expect = float(np.dot(x.cpu().numpy(), y.cpu().numpy()))
    assert got == pytest.approx(expect, rel=1e-12)


def test_dot_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    L = _lib.lib()
    dev = torch.device("cuda:0")
    buf = torch.zeros(2, dtype=torch.float64, device=dev)
    p = C.c_void_p(buf.data_ptr())
    assert L.chidg_gpu_dot_noalloc(0, p, p, MAX_N + 1, p, None) == _lib.EINVAL
    assert L.chidg_gpu_dot_noalloc(0, p, p, -1, p, None) == _lib.EINVAL
