"""The C++ stage API (include/mcnla_b200/isvd.hpp): it compiles here (CPU), and
on a GPU the reference's stage checks written against it pass
(tests/cpp/check_isvd.cpp)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out_dir, name="check_isvd"):
    exe = os.path.join(out_dir, name)
    lib_dir = os.path.join(ROOT, "mcnla_b200")
    cmd = ["g++", "-std=c++14", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o", exe,
           "-L", lib_dir, "-lmcnla_b200", "-Wl,-rpath," + lib_dir,
           "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_api_compiles(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    assert os.path.exists(build(str(tmp_path)))


def test_cpp_io_round_trips(tmp_path):
    """The C++ file API (mcnla_b200::io): host only, so it runs here."""
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    exe = build(str(tmp_path), "check_io")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")


@pytest.mark.gpu
def test_cpp_stage_checks_on_gpu(tmp_path, golden):
    exe = build(str(tmp_path))
    for name in ("qs", "ys", "qb_kn", "qb_wy", "a", "q", "u"):
        np.ascontiguousarray(golden[name], dtype="<f8").tofile(os.path.join(str(tmp_path), name + ".bin"))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK (0 failures)" in r.stdout
