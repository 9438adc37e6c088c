"""ctypes binding of ``libmcnla_b200.so`` (the C ABI in ``include/mcnla_b200.h``).

The library is the only compute path: when it is missing, or the machine has no
CUDA device, calls raise ``RuntimeError``.  There is no CPU fallback.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmcnla_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "mcnla_b200.h")

OK = 0
ERR_SHAPE, ERR_LAYOUT, ERR_WORKSPACE, ERR_CUDA, ERR_NOMEM, ERR_ARG, ERR_UNSUPPORTED, ERR_SINGULAR, \
    ERR_DEVICE_TIMEOUT, ERR_IO = range(1, 11)

ROW_MAJOR, COL_MAJOR = 0, 1

KOLMOGOROV_NAGUMO = 0
ROW_BLOCK_KOLMOGOROV_NAGUMO = 1
ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO = 2
ROW_BLOCK_WEN_YIN = 3
ROW_BLOCK_GRAMIAN_WEN_YIN = 4

SVD_FORMER = 0
GRAMIAN_FORMER = 1
ROW_BLOCK_GRAMIAN_FORMER = 2
COL_BLOCK_GRAMIAN_FORMER = 3

KN_AUTO, KN_EIGEN, KN_NEWTON_SCHULZ = 0, 1, 2

MAX_DIM_SKETCH = 160
MAX_DIM_SKETCH_WENYIN = 80


class Params(ctypes.Structure):
    """mirror of ``mcnla_b200_params``"""
    _fields_ = [("nrow", ctypes.c_int64), ("ncol", ctypes.c_int64), ("rank", ctypes.c_int64),
                ("over_rank", ctypes.c_int64), ("num_sketch", ctypes.c_int64)]


PRECISION_FP64, PRECISION_MIXED, PRECISION_MIXED3 = 0, 1, 2


class Problem(ctypes.Structure):
    """mirror of ``mcnla_b200_problem``"""
    _fields_ = [("params", Params), ("A", ctypes.c_void_p), ("A32", ctypes.c_void_p), ("a_layout", ctypes.c_int),
                ("lda", ctypes.c_int64), ("seed", ctypes.c_uint64), ("integrator", ctypes.c_int),
                ("former", ctypes.c_int), ("max_iteration", ctypes.c_int), ("tolerance", ctypes.c_double),
                ("precision", ctypes.c_int), ("S", ctypes.c_void_p), ("U", ctypes.c_void_p), ("V", ctypes.c_void_p),
                ("iteration", ctypes.c_int), ("status", ctypes.c_int), ("seconds", ctypes.c_double),
                ("latency", ctypes.c_double), ("a_hi", ctypes.c_void_p), ("a_lo", ctypes.c_void_p),
                ("a_lo2", ctypes.c_void_p), ("lda16", ctypes.c_int64), ("at_hi", ctypes.c_void_p),
                ("at_lo", ctypes.c_void_p), ("at_lo2", ctypes.c_void_p), ("ldat16", ctypes.c_int64)]


class McnlaError(RuntimeError):
    def __init__(self, status, what, detail=""):
        self.status = status
        msg = "%s failed: %s (status %d)" % (what, status_string(status), status)
        if detail:
            msg += ": " + detail
        super().__init__(msg)


_lib = None
_lock = threading.Lock()

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_INT = ctypes.c_int

# mcnla_b200_allreduce_fn: int (*)(void* user, double* buf, int64_t count, void* stream)
ALLREDUCE_FN = ctypes.CFUNCTYPE(_INT, _P, _P, _I64, _P)
READ_ROWS_FN = ctypes.CFUNCTYPE(_INT, _P, _I64, _I64, _P)
NCCL_ID_BYTES = 128

# name -> (restype, argtypes), one line per entry point of the header
SIGNATURES = {
    "mcnla_b200_set_allreduce": (_INT, [_P, ALLREDUCE_FN, _P]),
    "mcnla_b200_nccl_unique_id": (_INT, [_P]),
    "mcnla_b200_set_nccl": (_INT, [_P, _P, _INT, _INT]),
    "mcnla_b200_allreduces": (_I64, [_P]),
    "mcnla_b200_create": (_INT, [ctypes.POINTER(_P), _INT, _P]),
    "mcnla_b200_destroy": (_INT, [_P]),
    "mcnla_b200_set_stream": (_INT, [_P, _P]),
    "mcnla_b200_status_string": (ctypes.c_char_p, [_INT]),
    "mcnla_b200_mm_size": (_INT, [ctypes.c_char_p, ctypes.POINTER(_I64), ctypes.POINTER(_INT)]),
    "mcnla_b200_mm_load": (_INT, [ctypes.c_char_p, _I64, _I64, _I64, _I64, _P, _I64, _INT]),
    "mcnla_b200_mm_save": (_INT, [ctypes.c_char_p, _P, _I64, _I64, _I64, _I64, _INT, ctypes.c_char_p]),
    "mcnla_b200_binary_size": (_INT, [ctypes.c_char_p, ctypes.POINTER(_I64), ctypes.POINTER(_INT), ctypes.c_char_p]),
    "mcnla_b200_binary_load": (_INT, [ctypes.c_char_p, _I64, _I64, _P]),
    "mcnla_b200_binary_save": (_INT, [ctypes.c_char_p, _P, _INT, ctypes.POINTER(_I64), ctypes.c_char_p]),
    "mcnla_b200_last_error": (ctypes.c_char_p, []),
    "mcnla_b200_kernels_launched": (_I64, [_P]),
    "mcnla_b200_graph_replays": (_I64, [_P]),
    "mcnla_b200_set_kn_method": (_INT, [_P, _INT]),
    "mcnla_b200_set_autotune": (_INT, [_P, _INT]),
    "mcnla_b200_set_cta_limit": (_INT, [_P, _INT]),
    "mcnla_b200_set_graph_loop": (_INT, [_P, _INT]),
    "mcnla_b200_last_times": (_INT, [_P, ctypes.POINTER(_D), _INT]),
    "mcnla_b200_initialize": (_INT, [_P, ctypes.POINTER(Params), _INT, _INT]),
    "mcnla_b200_sketch": (_INT, [_P, ctypes.POINTER(Params), _P, _INT, _I64, _P, _INT, _P]),
    "mcnla_b200_gaussian": (_INT, [_P, ctypes.c_uint64, _I64, _P]),
    "mcnla_b200_orthogonalize": (_INT, [_P, ctypes.POINTER(Params), _P]),
    "mcnla_b200_integrate": (_INT, [_P, ctypes.POINTER(Params), _INT, _P, _INT, _D, _P, ctypes.POINTER(_INT)]),
    "mcnla_b200_form": (_INT, [_P, ctypes.POINTER(Params), _INT, _P, _INT, _I64, _P, _P, _P, _P]),
    "mcnla_b200_isvd": (_INT, [_P, ctypes.POINTER(Params), _INT, _INT, _P, _INT, _I64, _P, ctypes.c_uint64, _INT, _D,
                               _P, _P, _P, ctypes.POINTER(_INT)]),
    "mcnla_b200_isvd_host": (_INT, [_P, ctypes.POINTER(Params), _INT, _INT, _P, _INT, _P, _INT, _D, _P, _P, _P,
                                    ctypes.POINTER(_INT)]),
    "mcnla_b200_isvd_stream": (_INT, [_P, ctypes.POINTER(Params), _INT, _INT, READ_ROWS_FN, _P, _P, _INT, _D, _P, _P,
                                      _P, ctypes.POINTER(_INT)]),
    "mcnla_b200_dgemm": (_INT, [_P, _I64, _I64, _I64, _D, _P, _I64, _I64, _P, _I64, _I64, _D, _P, _I64, _I64, _INT]),
    "mcnla_b200_syev_batched": (_INT, [_P, _INT, _INT, _P, _P, _P, _INT]),
    "mcnla_b200_inverse_batched": (_INT, [_P, _INT, _INT, _P]),
    "mcnla_b200_split_bf16": (_INT, [_P, _P, _INT, _I64, _I64, _I64, _P, _P, _P, _I64]),
    "mcnla_b200_gaussian_bf16": (_INT, [_P, ctypes.c_uint64, _I64, _I64, _P, _I64, _P]),
    "mcnla_b200_gemm_bf16": (_INT, [_P, _I64, _I64, _I64, _P, _P, _P, _I64, _P, _I64, _P, _I64, _INT]),
    "mcnla_b200_sketch_bf16": (_INT, [_P, ctypes.POINTER(Params), _P, _P, _P, _I64, _P, _I64, _P]),
    "mcnla_b200_form_bf16": (_INT, [_P, ctypes.POINTER(Params), _INT, _P, _P, _P, _I64, _P, _P, _P, _P]),
    "mcnla_b200_isvd_mixed": (_INT, [_P, ctypes.POINTER(Params), _INT, _INT, _P, _INT, _I64, _P, _P, _P, _I64,
                                     _P, _P, _P, _I64, ctypes.c_uint64, _INT, _D, _P, _P, _P,
                                     ctypes.POINTER(_INT)]),
    "mcnla_b200_problem_bytes": (_I64, [ctypes.POINTER(Problem)]),
    "mcnla_b200_server_create": (_INT, [ctypes.POINTER(_P), _INT, _INT, _I64]),
    "mcnla_b200_server_submit": (_INT, [_P, ctypes.POINTER(Problem), ctypes.POINTER(_I64)]),
    "mcnla_b200_server_wait": (_INT, [_P, _I64, ctypes.POINTER(Problem)]),
    "mcnla_b200_server_stats": (_INT, [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    "mcnla_b200_server_destroy": (_INT, [_P]),
    "mcnla_b200_isvd_batched": (_INT, [_INT, ctypes.POINTER(Problem), _INT, _INT, _I64]),
    "mcnla_b200_isvd_grouped": (_INT, [_INT, ctypes.POINTER(Problem), _INT, _INT, _I64]),
    "mcnla_b200_grouped_times": (_INT, [ctypes.POINTER(_D), _INT]),
    "mcnla_b200_dgemm_noalloc": (_INT, [_P, _I64, _I64, _I64, _D, _P, _I64, _I64, _P, _I64, _I64, _D, _P, _I64,
                                        _I64]),
}


def load():
    """Loads the library (once) and declares every entry point."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError("mcnla_b200: %s is missing; build it with `python -m mcnla_b200.build`" % LIB_PATH)
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def status_string(status):
    try:
        return load().mcnla_b200_status_string(status).decode()
    except Exception:  # the library itself may be what is missing
        return "status %d" % status


def check(status, what):
    if status != OK:
        detail = ""
        if status == ERR_CUDA:
            detail = load().mcnla_b200_last_error().decode()
        raise McnlaError(status, what, detail)
    return status
