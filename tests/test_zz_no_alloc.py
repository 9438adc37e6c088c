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
