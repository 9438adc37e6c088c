"""CPU checks of the C ABI: the library loads, exports every entry point the
header declares, and the Python binding declares each one.  No compute call is
made (this machine may have no GPU)."""
import ctypes
import os
import re
import subprocess

import pytest

from mcnla_b200 import _lib


def declared_symbols():
    text = open(_lib.HEADER_PATH).read()
    return sorted(set(re.findall(r"MCNLA_B200_API\s+[\w\s\*]+?\b(mcnla_b200_\w+)\s*\(", text)))


def test_library_present():
    assert os.path.exists(_lib.LIB_PATH), "build it: python -m mcnla_b200.build"


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 18
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (mcnla_b200_\w+)", out))
    assert set(syms) == exported, (set(syms) ^ exported)


def test_binding_declares_every_symbol():
    assert sorted(_lib.SIGNATURES) == declared_symbols()
    _lib.load()


def test_status_strings():
    lib = _lib.load()
    assert lib.mcnla_b200_status_string(0) == b"ok"
    for st in range(1, 10):
        assert lib.mcnla_b200_status_string(st) != b"unknown status"
    assert lib.mcnla_b200_status_string(99) == b"unknown status"


def test_header_constants_match_binding():
    text = open(_lib.HEADER_PATH).read()
    consts = dict((k, int(v)) for k, v in re.findall(r"#define (MCNLA_B200_\w+)\s+(\d+)", text))
    assert consts["MCNLA_B200_ROW_BLOCK_GRAMIAN_WEN_YIN"] == _lib.ROW_BLOCK_GRAMIAN_WEN_YIN
    assert consts["MCNLA_B200_COL_BLOCK_GRAMIAN_FORMER"] == _lib.COL_BLOCK_GRAMIAN_FORMER
    assert consts["MCNLA_B200_MAX_DIM_SKETCH"] == _lib.MAX_DIM_SKETCH
    assert consts["MCNLA_B200_ERR_SINGULAR"] == _lib.ERR_SINGULAR


def test_null_arguments_are_rejected_without_device_work():
    lib = _lib.load()
    assert lib.mcnla_b200_create(None, 0, None) == _lib.ERR_ARG
    assert lib.mcnla_b200_destroy(None) == _lib.OK
    p = _lib.Params(10, 10, 2, 2, 2)
    assert lib.mcnla_b200_integrate(None, ctypes.byref(p), 0, None, 1, 1e-4, None, None) == _lib.ERR_ARG
    assert lib.mcnla_b200_form(None, ctypes.byref(p), 0, None, 0, 10, None, None, None, None) == _lib.ERR_ARG


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.mcnla_b200_create(ctypes.byref(h), 0, None)
    assert st == _lib.ERR_CUDA
    assert not h.value
    assert lib.mcnla_b200_last_error()


def test_header_is_plain_c(tmp_path):
    """include/mcnla_b200.h is a C header (C99, no warnings under -Wall -Wextra -pedantic) and
    a C program links the library and calls it (host-only entry points: no GPU needed)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no gcc")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "abi_check.c"
    src.write_text(
        "#include <mcnla_b200.h>\n#include <stdio.h>\n"
        "int main(void) {\n"
        "  int64_t dims[3]; int nd = 0;\n"
        "  printf(\"%s\\n\", mcnla_b200_status_string(MCNLA_B200_ERR_IO));\n"
        "  return mcnla_b200_mm_size(\"/nonexistent/x.mtx\", dims, &nd) == MCNLA_B200_ERR_IO ? 0 : 1;\n"
        "}\n")
    exe = tmp_path / "abi_check"
    lib_dir = os.path.join(root, "mcnla_b200")
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                        os.path.join(root, "include"), str(src), "-o", str(exe), "-L", lib_dir, "-lmcnla_b200",
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "file" in r.stdout
