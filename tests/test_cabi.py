"""The C ABI library loads and exports every entry point of include/chidg_gpu.h
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import numpy as np

from chidg_b200 import _lib, mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(chidg_gpu_\w+)\s*\(", text)))


def test_header_symbols_exported():
    names = header_functions(os.path.join(ROOT, "include", "chidg_gpu.h"))
    assert len(names) >= 40
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header():
    names = header_functions(os.path.join(ROOT, "include", "chidg_gpu.h"))
    assert set(names) <= set(_lib.PROTOTYPES), set(names) - set(_lib.PROTOTYPES)


def test_struct_layouts():
    # the ctypes mirrors must match the C structs field for field
    assert ctypes.sizeof(_lib.Pattern) == 8 + 8 * 3 + 8 + 8 * 5
    assert ctypes.sizeof(_lib.FgmresResult) == 4 * 4 + 8 * 4


def test_box_pattern_matches_reference_layout():
    # 3x1x1: element 1 has [XI_MAX, DIAG], element 2 [XI_MIN, XI_MAX, DIAG], element 3 [XI_MIN, DIAG]
    pat = mesh.box_pattern(3, 1, 1, 1, 1)
    assert pat.blk_row_elem.tolist() == [0, 0, 1, 1, 1, 2, 2]
    assert pat.blk_col_elem.tolist() == [1, 0, 0, 2, 1, 1, 2]
    # 24^3 P2 (the 13.6 GB FP64 workload): 93 312 blocks of 135 x 135
    pat = mesh.box_pattern(24, 24, 24, 5, mesh.nterms_of_order(2))
    assert pat.nblocks == 93312
    _, nval = pat.value_offsets()
    assert nval * 8 == 13_604_889_600
    assert int((pat.blk_col_elem < pat.blk_row_elem).sum()) == 39744


def test_box_pattern_hb_and_subdomains():
    pat = mesh.box_pattern(2, 2, 2, 5, 8, ntime=3, subdomains=(2, 2, 2))
    assert sorted(set(pat.elem_proc.tolist())) == list(range(8))
    hb = pat.blk_kind == _lib.BLK_HB
    assert hb.sum() == 8 * 3 * 2
    assert np.all(pat.blk_row_elem[hb] == pat.blk_col_elem[hb])
    assert np.all(pat.blk_row_time[hb] != pat.blk_col_time[hb])


def test_synth_is_deterministic_and_thread_independent():
    pat = mesh.box_pattern(3, 2, 2, 5, 8)
    a = mesh.synth_values(pat, seed=1, nthreads=1)
    b = mesh.synth_values(pat, seed=1, nthreads=4)
    c = mesh.synth_values(pat, seed=2, nthreads=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)


def test_selftest_argument_checks_need_no_gpu():
    """The self-test entry refuses bad arguments before touching the device."""
    import ctypes as C
    from chidg_b200 import _lib
    L = _lib.lib()
    bits = C.c_int32(0)
    assert L.chidg_gpu_selftest_bounded_waits(None, 1000, C.byref(bits)) == _lib.EINVAL
