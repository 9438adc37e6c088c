"""ctypes binding of the reference checker ``oracle/_ref/libmcnla_ref.so``.

Test infrastructure: only tests, the smoke check and the bench's CPU-baseline
leg use it.  The library is the reference's own stages (built by
``make -C oracle`` from the reference headers); see ``oracle/ref/ref_harness.cpp``
for the conventions of each entry point.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libmcnla_ref.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def available():
    return os.path.exists(LIB_PATH)


def load():
    lib = ctypes.CDLL(LIB_PATH)
    lib.mref_sketch.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, _D, _D]
    # every `t` argument points at 8 doubles: time() then the parts of times()
    lib.mref_orthogonalize.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D]
    lib.mref_integrate.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, _D, _I, _D]
    lib.mref_form.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int, _D, _D, _D, _D]
    lib.mref_solver_create.restype = ctypes.c_void_p
    lib.mref_solver_create.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, _D]
    lib.mref_solver_run.argtypes = [ctypes.c_void_p, _D, _I]
    lib.mref_solver_result.argtypes = [ctypes.c_void_p, _D, _D, _D]
    lib.mref_solver_destroy.argtypes = [ctypes.c_void_p]
    lib.mref_set_threads.argtypes = [ctypes.c_int]
    lib.mref_get_threads.restype = ctypes.c_int
    return lib


def _p(a):
    return a.ctypes.data_as(_D)


def _c(a, order="C"):
    return np.require(a, dtype=np.float64, requirements=[order, "A"])


def _times():
    return np.zeros(8)


def sketch(lib, a, omega, colmajor=False):
    """Returns (Y, seconds of the GEMM)."""
    m, n = a.shape
    L = omega.shape[1]
    ab = _c(a.T if colmajor else a)          # column-major A == row-major A^T buffer
    om = _c(omega)
    y = np.empty((m, L))
    t = _times()
    lib.mref_sketch(_p(ab), int(colmajor), m, n, _p(om), L, _p(y), _p(t))
    return y, t[0]


def orthogonalize(lib, y, l, N, row_block=False, timing=False, inplace=False):
    """timing=True also returns [time(), parts...].  inplace=True orthogonalizes y
    itself (a C-contiguous float64 array) instead of a copy."""
    q = y if inplace and y.flags.c_contiguous and y.dtype == np.float64 else _c(y).copy()
    m = q.shape[0]
    t = _times()
    lib.mref_orthogonalize(_p(q), m, l, N, int(row_block), _p(t))
    return (q, t) if timing else q


def integrate(lib, qs, l, N, kind, maxit, tol, timing=False):
    qs = _c(qs)
    m = qs.shape[0]
    qbar = np.empty((m, l))
    it = ctypes.c_int()
    t = _times()
    rc = lib.mref_integrate(_p(qs), m, l, N, kind, maxit, tol, _p(qbar), ctypes.byref(it), _p(t))
    assert rc == 0
    return (qbar, it.value, t) if timing else (qbar, it.value)


def form(lib, a, qbar, k, p, kind, colmajor=False, timing=False):
    m, n = a.shape
    ab = _c(a.T if (colmajor or kind == 3) else a)
    qb = _c(qbar)
    s = np.empty(k)
    u = np.empty((m, k))
    v = np.empty((n, k))
    t = _times()
    rc = lib.mref_form(_p(ab), int(colmajor or kind == 3), m, n, _p(qb), k, p, kind, _p(s), _p(u), _p(v), _p(t))
    assert rc == 0
    return (s, u, v, t) if timing else (s, u, v)


class Solver:
    """A whole reference solve held between runs (mref_solver_*): A and Omega are loaded into
    the reference's own matrices and the four stages constructed and initialized once, as the
    reference's drivers do before they time anything; run() executes sketch -> orthogonalize ->
    integrate -> form and returns (iterations, [sketch, orthogonalize, integrate, form] seconds
    from the stages' own timers).  kind / fkind: as integrate() / form()."""

    def __init__(self, lib, a, omega, k, p, N, kind, fkind, maxit, tol, colmajor=False, row_block=True):
        m, n = a.shape
        self.lib, self.k, self.m, self.n = lib, k, m, n
        ab = _c(a.T if colmajor else a)
        om = _c(omega)
        self.h = lib.mref_solver_create(_p(ab), int(colmajor), m, n, k, p, N, int(row_block), kind, fkind, maxit,
                                        tol, _p(om))
        if not self.h:
            raise ValueError("unsupported integrator / former / layout combination")

    def run(self):
        t = np.zeros(4)
        it = ctypes.c_int()
        assert self.lib.mref_solver_run(self.h, _p(t), ctypes.byref(it)) == 0
        return it.value, t

    def result(self):
        s, u, v = np.empty(self.k), np.empty((self.m, self.k)), np.empty((self.n, self.k))
        assert self.lib.mref_solver_result(self.h, _p(s), _p(u), _p(v)) == 0
        return s, u, v

    def close(self):
        if self.h:
            self.lib.mref_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
