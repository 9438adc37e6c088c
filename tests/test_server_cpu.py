"""CPU checks of the server's admission estimate (mcnla_b200_problem_bytes, host only): the
device bytes a problem is admitted with, including the precision form's buffers."""
import ctypes

from mcnla_b200 import _lib


def _bytes(m, n, k, p, N, precision, integrator, fp32=True, resident=False):
    pr = _lib.Problem()
    pr.params = _lib.Params(m, n, k, p, N)
    pr.A = None if fp32 else ctypes.c_void_p(0x1000)
    pr.A32 = ctypes.c_void_p(0x1000) if fp32 else None   # only their presence is read
    pr.integrator = integrator
    pr.precision = precision
    if resident:                                          # the caller's BF16 parts of A and A'
        pr.a_hi = pr.a_lo = pr.a_lo2 = pr.at_hi = pr.at_lo = pr.at_lo2 = ctypes.c_void_p(0x2000)
    return _lib.load().mcnla_b200_problem_bytes(ctypes.byref(pr))


def r8(x):
    return (x + 7) & ~7


def test_precision_form_parts_and_fp64_copy():
    m, n, k, p, N = 8192, 2048, 32, 16, 8
    g = _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO
    fp64 = _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g)
    mixed3 = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, g)
    L = (k + p) * N
    # mixed: Omega' in BF16 instead of the FP64 Omega, three BF16 parts of A (sketch) and of A'
    # (precision former) instead of the FP64 copy of the FP32 A; (N l)^2 m = 1.5e9 < 1e11: no
    # BF16 Gramian; the stage workspaces are the same here
    assert mixed3 - fp64 == L * r8(n) * 2 - n * L * 8 + 3 * m * r8(n) * 2 + 3 * n * r8(m) * 2 - m * n * 8
    assert fp64 - _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g, fp32=False) == m * n * 8
    # resident parts: nothing is split per request
    assert mixed3 - _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, g, resident=True) == \
        3 * m * r8(n) * 2 + 3 * n * r8(m) * 2


def test_large_mixed_gramian_scratch_counted():
    m, n, k, p, N = 65536, 8192, 128, 32, 16          # the large served request: (N l)^2 m = 4.3e11
    l, L = k + p, (k + p) * N
    g = _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO
    with_gramian = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, g)
    plain_kn = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, _lib.KOLMOGOROV_NAGUMO)
    extra = 3 * L * r8(m) * 2 + 3 * L * r8(L) * 2 + 3 * l * r8(L) * 2 + 16 * L * 3 * l * 8
    assert with_gramian - plain_kn == extra
    assert extra > 1 << 30
    # the Wen-Yin Gramian integrator takes only the parts of Qs' (no Bs Bc loop product)
    wy = _bytes(m, n, k, p, N, _lib.PRECISION_MIXED3, _lib.ROW_BLOCK_GRAMIAN_WEN_YIN)
    assert wy - plain_kn == 3 * L * r8(m) * 2
    # FP64 solves never take the BF16 Gramian
    assert _bytes(m, n, k, p, N, _lib.PRECISION_FP64, g) == _bytes(m, n, k, p, N, _lib.PRECISION_FP64,
                                                                    _lib.KOLMOGOROV_NAGUMO)


def test_null_problem():
    assert _lib.load().mcnla_b200_problem_bytes(None) == -1
