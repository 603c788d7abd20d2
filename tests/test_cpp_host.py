"""The C++ host layer (include/chidg_gpu.hpp): it compiles and links against
the library (CPU), and replays the reference's known-answer tests on the GPU."""
import os
import subprocess

import pytest

from tests import kat_util

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(ROOT, "chidg_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "test_reference_kats.cpp")


EULER_SRC = os.path.join(ROOT, "tests", "cpp", "test_euler_freestream.cpp")
BATCH_SRC = os.path.join(ROOT, "tests", "cpp", "test_batched_serve.cpp")


def build(tmp_path, src=SRC):
    if not os.path.exists(os.path.join(LIB_DIR, "libchidg_gpu.so")):
        pytest.skip("libchidg_gpu.so is not built")
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), src,
                           "-o", exe, "-L", LIB_DIR, "-lchidg_gpu", "-Wl,-rpath," + LIB_DIR])
    return exe


def cases_text():
    out = []
    for name in ("ilu0", "ilu0_hb", "fgmres", "fgmres_ref"):
        c = kat_util.load_cases()[name]
        out.append(f"case {name} {c['nelem_xi']} {c['ntime']} {c['tol'] or 0.0!r} {c['solver_tol'] or 0.0!r}")
        out += [f"block {e} {t} {col} {v!r}" for e, t, col, v in c["blocks"]]
        out += [f"rhs {e} {v!r}" for e, v in c["rhs"]]
        for kind, idx, v in c["asserts"]:
            out.append(f"{kind} {' '.join(str(i) for i in idx)} {v!r}")
        out.append("end")
    return "\n".join(out) + "\n"


def test_host_layer_compiles_and_links(tmp_path):
    assert os.path.exists(build(tmp_path))
    assert os.path.exists(build(tmp_path, EULER_SRC))
    assert os.path.exists(build(tmp_path, BATCH_SRC))


@pytest.mark.gpu
def test_reference_kats_through_cpp_host_layer(tmp_path):
    exe = build(tmp_path)
    cases = tmp_path / "cases.txt"
    cases.write_text(cases_text())
    p = subprocess.run([exe, str(cases)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "4 cases, 0 failures" in p.stdout


@pytest.mark.gpu
def test_euler_assembly_through_cpp_host_layer(tmp_path):
    exe = build(tmp_path, EULER_SRC)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr


@pytest.mark.gpu
def test_batched_and_served_solves_through_cpp_host_layer(tmp_path):
    exe = build(tmp_path, BATCH_SRC)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "0 failures" in p.stdout
