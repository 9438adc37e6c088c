"""Builds the in-tree shared library ``mcnla_b200/libmcnla_b200.so`` for sm_100a.

The library is plain CUDA C++ behind the C ABI of ``include/mcnla_b200.h``; no
torch headers are involved.  Usage::

    python -m mcnla_b200.build            # or: python mcnla_b200/build.py
"""
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmcnla_b200.so")
BUILD_DIR = os.path.join(ROOT, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "mcnla_b200.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=True, jobs=None):
    """Compiles each .cu to an object (in parallel) and links the .so.  Skips
    work that is up to date.  Returns the library path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    hdrs = _headers()
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    t0 = time.time()
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors="replace")))
        elif verbose and out.strip():
            sys.stdout.write(out.decode(errors="replace"))
    if failed:
        for src, out in failed:
            sys.stderr.write("---- %s\n%s\n" % (src, out))
        raise RuntimeError("nvcc failed for: " + ", ".join(os.path.basename(s) for s, _ in failed))
    if _stale(LIB, objs):
        cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs]
        subprocess.run(cmd, check=True)
    if verbose:
        print("built %s (%d objects, %.1fs)" % (LIB, len(objs), time.time() - t0))
    return LIB


if __name__ == "__main__":
    build()
