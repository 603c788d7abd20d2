"""Matrices to and from files: chidg_matrix%to_file's text listing against
the oracle's restatement (byte for byte, values in every branch of the
F24.14 / E24.14 choice), and the binary image's save / load round trip."""
import numpy as np
import pytest

from chidg_b200 import _lib, api, mesh
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def spread_values(pat, seed):
    """Synthetic values scaled over many decades, with exact 0, 0.1 and 1e9."""
    rng = np.random.default_rng(seed)
    v = mesh.synth_values(pat, seed=seed)
    v *= 10.0 ** rng.integers(-130, 13, size=v.size)
    v[::17] = 0.0
    v[5::23] = 0.1
    v[7::29] = -1e9
    v[9::31] = -123456789.25          # too wide for F24.14: asterisks
    return v


@pytest.mark.parametrize("shape,P,nvars,nt", [((2, 2, 1), 1, 2, 1), ((2, 1, 1), 0, 3, 2)])
def test_to_file_matches_oracle(tmp_path, shape, P, nvars, nt):
    pat = mesh.box_pattern(*shape, nvars, mesh.nterms_of_order(P), ntime=nt)
    vals = spread_values(pat, seed=71)
    A = api.ChidgMatrix(pat)
    A.upload(vals)
    path = tmp_path / "matrix.txt"
    A.to_file(str(path))
    assert path.read_text() == O.to_file_text(pat, vals)


def test_save_load_round_trip(tmp_path):
    pat = mesh.box_pattern(3, 2, 2, 5, mesh.nterms_of_order(1), ntime=2)
    vals = mesh.synth_values(pat, seed=73)
    A = api.ChidgMatrix(pat)
    A.upload(vals)
    A.transposed = True
    path = tmp_path / "matrix.bin"
    A.save(str(path))
    B = api.ChidgMatrix.load(str(path))
    assert B.transposed
    assert np.array_equal(B.download(), vals)
    for f in ("elem_nvars", "elem_nterms", "elem_proc", "blk_row_elem", "blk_row_time", "blk_col_elem",
              "blk_col_time", "blk_kind"):
        assert np.array_equal(getattr(B.pattern, f), getattr(pat, f)), f
    x = mesh.synth_vector(pat.vector_size(), seed=74)
    ya = api.chidg_mv(A, api.ChidgVector(A, x)).download()
    yb = api.chidg_mv(B, api.ChidgVector(B, x)).download()
    assert np.array_equal(ya, yb)


def test_load_rejects_bad_files(tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTAMATRIX" + bytes(64))
    with pytest.raises(_lib.ChidgGpuError) as ei:
        api.ChidgMatrix.load(str(bad))
    assert ei.value.code == _lib.EINVAL
    pat = mesh.box_pattern(2, 2, 1, 2, mesh.nterms_of_order(1))
    A = api.ChidgMatrix(pat)
    A.upload(mesh.synth_values(pat, seed=75))
    good = tmp_path / "good.bin"
    A.save(str(good))
    cut = tmp_path / "cut.bin"
    cut.write_bytes(good.read_bytes()[:-8])
    with pytest.raises(_lib.ChidgGpuError) as ei:
        api.ChidgMatrix.load(str(cut))
    assert ei.value.code == _lib.EINVAL
    with pytest.raises(_lib.ChidgGpuError):
        api.ChidgMatrix.load(str(tmp_path / "missing.bin"))
