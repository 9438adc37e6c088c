"""The FP64 GEMM entry point that allocates nothing (mcnla_b200_dgemm_noalloc).

It serves callers that cannot call cudaMalloc (a plugin whose host framework
owns the device memory pool; a latency-critical loop that cannot take an
allocation's implicit synchronization): its split-K partial sums live in a
fixed 16 MiB device array of the library instead of a context workspace.
This file is collected last so that, should it fail, a run that stops at the
first failure has run every other test already.  Each test checks the
entry point against mcnla_b200_dgemm (which allocates its workspace) on two
calls in a row, with the tolerance of the GEMM parity tests.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu

# long-K products like the stages' Gram and reduction GEMMs (split-K used), an
# odd leading dimension, transposed operands and a shape with no split
SHAPES = [(64, 64, 100000, False, False), (20, 20, 100000, True, False), (101, 11, 1001, False, True),
          (128, 128, 60000, True, True), (300, 200, 50, False, False)]


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _operands(M, N, K, ta, tb, dev, seed):
    g = torch.Generator(device=dev).manual_seed(seed)
    a = torch.randn(K, M, generator=g, dtype=torch.float64, device=dev).t() if ta else \
        torch.randn(M, K, generator=g, dtype=torch.float64, device=dev)
    b = torch.randn(N, K, generator=g, dtype=torch.float64, device=dev).t() if tb else \
        torch.randn(K, N, generator=g, dtype=torch.float64, device=dev)
    c0 = torch.randn(M, N, generator=g, dtype=torch.float64, device=dev)
    return a, b, c0


@pytest.mark.parametrize("M,N,K,ta,tb", SHAPES)
def test_noalloc_matches_workspace_gemm(M, N, K, ta, tb):
    from mcnla_b200 import _lib, isvd
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    ctx = isvd.context(dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    a, b, c0 = _operands(M, N, K, ta, tb, dev, M + N + K)
    alpha, beta = 0.75, -1.5
    ref = c0.clone()
    _lib.check(lib.mcnla_b200_dgemm(ctx.bind(), M, N, K, alpha, _p(a), a.stride(0), a.stride(1), _p(b),
                                    b.stride(0), b.stride(1), beta, _p(ref), ref.stride(0), ref.stride(1), 0),
               "dgemm")
    scale = (a.abs() @ b.abs()).max().item() * abs(alpha) + c0.abs().max().item() * abs(beta)
    tol = 1e-14 * scale * max(1, K) ** 0.5
    for call in range(2):          # two calls in a row share the static scratch
        c = c0.clone()
        _lib.check(lib.mcnla_b200_dgemm_noalloc(stream, M, N, K, alpha, _p(a), a.stride(0), a.stride(1), _p(b),
                                                b.stride(0), b.stride(1), beta, _p(c), c.stride(0), c.stride(1)),
                   "dgemm_noalloc")
        torch.cuda.synchronize()
        assert (c - ref).abs().max().item() <= tol, call
        exact = alpha * (a @ b) + beta * c0
        assert (c - exact).abs().max().item() <= tol, call


def test_noalloc_rejects_partials_beyond_the_scratch():
    from mcnla_b200 import _lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    M = N = 512
    K = 100000                     # split-K partials of 19 x 512 x 512 doubles: 38 MiB
    a, b, c = _operands(M, N, K, False, False, dev, 7)
    before = c.clone()
    st = lib.mcnla_b200_dgemm_noalloc(stream, M, N, K, 1.0, _p(a), K, 1, _p(b), N, 1, 0.0, _p(c), N, 1)
    assert st == _lib.ERR_SHAPE
    assert b"static scratch" in lib.mcnla_b200_last_error()
    torch.cuda.synchronize()
    assert torch.equal(c, before)


def test_noalloc_leaves_device_free_memory_unchanged():
    """The property the entry point exists for: after the first call (which may load the
    library's module), a call takes no device memory, and neither does a second one."""
    from mcnla_b200 import _lib
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    M, N, K = 128, 128, 60000      # split-K: the partial sums go to the static scratch
    a, b, c = _operands(M, N, K, False, False, dev, 11)

    def call():
        _lib.check(lib.mcnla_b200_dgemm_noalloc(stream, M, N, K, 1.0, _p(a), K, 1, _p(b), N, 1, 0.0, _p(c), N, 1),
                   "dgemm_noalloc")
        torch.cuda.synchronize()

    call()
    free0, _ = torch.cuda.mem_get_info(dev)
    call()
    free1, _ = torch.cuda.mem_get_info(dev)
    call()
    free2, _ = torch.cuda.mem_get_info(dev)
    assert free0 == free1 == free2, (free0, free1, free2)
    assert (c - a @ b).abs().max().item() <= 1e-14 * (a.abs() @ b.abs()).max().item() * K ** 0.5


_FRESH = r"""
import ctypes, sys, torch
sys.path.insert(0, sys.argv[1])
from mcnla_b200 import _lib
lib = _lib.load()
dev = torch.device("cuda", 0)
g = torch.Generator(device=dev).manual_seed(5)
M, N, K = 96, 80, 50000
a = torch.randn(M, K, generator=g, dtype=torch.float64, device=dev)
b = torch.randn(K, N, generator=g, dtype=torch.float64, device=dev)
c = torch.empty(M, N, dtype=torch.float64, device=dev)
torch.cuda.synchronize()
P = lambda t: ctypes.c_void_p(t.data_ptr())
for call in range(2):
    c.zero_()
    torch.cuda.synchronize()
    st = lib.mcnla_b200_dgemm_noalloc(None, M, N, K, 1.0, P(a), K, 1, P(b), N, 1, 0.0, P(c), N, 1)
    assert st == 0, (st, lib.mcnla_b200_last_error())
    torch.cuda.synchronize()
    tol = 1e-14 * (a.abs() @ b.abs()).max().item() * K ** 0.5
    err = (c - a @ b).abs().max().item()
    assert err <= tol, (call, err, tol)
print("fresh ok")
"""


def test_noalloc_first_call_in_a_fresh_process_on_the_null_stream():
    """The documented use: a caller that never creates a library context makes its first call
    on a device with the NULL (default) stream; checked against torch's a @ b."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FRESH, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
