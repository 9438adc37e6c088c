"""CPU checks of the server's admission estimate (mcnla_b200_problem_bytes, host only): the
device bytes a problem is admitted with, including the precision form's buffers."""
import ctypes

from mcnla_b200 import _lib


def _bytes(m, n, k, p, N, precision, integrator, fp32=True):
    pr = _lib.Problem()
    pr.params = _lib.Params(m, n, k, p, N)
    pr.A = None
    pr.A32 = ctypes.c_void_p(0x1000) if fp32 else None   # only its presence is read
    pr.integrator = integrator
    pr.precision = precision
    return _lib.load().mcnla_b200_problem_bytes(ctypes.byref(pr))


def r8(x):
    return (x + 7) & ~7


def test_precision_form_parts_and_fp64_copy():
    m, n, k, p, N = 8192, 2048, 32, 16, 8
    g = _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO
    fp64 = _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g)
    mixed3 = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, g)
    L = (k + p) * N
    # three BF16 parts of A and Omega' in BF16; (N l)^2 m = 1.5e9 < 1e11: no BF16 Gramian
    assert mixed3 - fp64 == 3 * m * r8(n) * 2 + L * r8(n) * 2
    assert fp64 - _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g, fp32=False) == m * n * 8


def test_large_mixed_gramian_scratch_counted():
    m, n, k, p, N = 65536, 8192, 128, 32, 16          # the large served request: (N l)^2 m = 4.3e11
    l, L = k + p, (k + p) * N
    g = _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO
    with_gramian = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, g)
    plain_kn = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, _lib.KOLMOGOROV_NAGUMO)
    extra = 3 * L * r8(m) * 2 + 3 * L * r8(L) * 2 + 3 * l * r8(L) * 2 + 16 * L * 3 * l * 8
    assert with_gramian - plain_kn == extra
    assert extra > 1 << 30
    # FP64 solves never take the BF16 Gramian
    assert _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g) == _bytes(m, n, k, p, N, _lib.PRECISION_FP64,
                                                                    _lib.KOLMOGOROV_NAGUMO)


def test_null_problem():
    assert _lib.load().mcnla_b200_problem_bytes(None) == -1
