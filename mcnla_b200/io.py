"""Dense files of the reference's io module (include/mcnla/core/io/): MatrixMarket "array"
text and the MCNLA dense binary format, read and written by the library's host code
(csrc/io.cu, ``mcnla_b200_mm_*`` / ``mcnla_b200_binary_*``), plus the copy of a loaded
matrix to the device through pinned memory.

A 3-D MatrixMarket collection (l matrices of m x n) is handled as its unfolded m x (n l)
matrix, matrix k in columns [k n, (k + 1) n): the layout of the sketch collection Q."""
import ctypes

import numpy as np

from . import _lib

ROW_MAJOR, COL_MAJOR = _lib.ROW_MAJOR, _lib.COL_MAJOR


def _path(p):
    return str(p).encode()


def matrix_market_size(path):
    """(m, n, l) of a dense MatrixMarket file (l = 1 for a matrix)."""
    dims = (ctypes.c_int64 * 3)()
    nd = ctypes.c_int()
    _lib.check(_lib.load().mcnla_b200_mm_size(_path(path), dims, ctypes.byref(nd)), "mm_size")
    return tuple(int(d) for d in dims)


def load_matrix_market(path, rows=None, cols=None, order="C"):
    """The (unfolded) matrix of a dense MatrixMarket file as float64, or the block
    rows = (first, count) x cols = (first, count) of it (loadMatrixMarketRowBlock /
    ColBlock).  order "C" gives a row-major array, "F" a column-major one."""
    m, n, l = matrix_market_size(path)
    r0, nr = rows if rows is not None else (0, m)
    c0, nc = cols if cols is not None else (0, n * l)
    out = np.empty((nr, nc), dtype=np.float64, order=order)
    layout = ROW_MAJOR if order == "C" else COL_MAJOR
    ld = nc if order == "C" else nr
    _lib.check(_lib.load().mcnla_b200_mm_load(_path(path), r0, nr, c0, nc,
                                              out.ctypes.data_as(ctypes.c_void_p), max(ld, 1), layout), "mm_load")
    return out


def save_matrix_market(path, a, nmat=1, comment=None):
    """Writes a 2-D array (m x (n nmat), the unfolded collection when nmat > 1) as the
    reference's saveMatrixMarket does."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] % nmat:
        raise ValueError("a must be m x (n nmat)")
    if not (a.flags.c_contiguous or a.flags.f_contiguous):
        a = np.ascontiguousarray(a)
    layout = ROW_MAJOR if a.flags.c_contiguous else COL_MAJOR
    m, cols = a.shape
    ld = max(cols if layout == ROW_MAJOR else m, 1)
    _lib.check(_lib.load().mcnla_b200_mm_save(_path(path), a.ctypes.data_as(ctypes.c_void_p), m, cols // nmat, nmat,
                                              ld, layout, comment.encode() if comment else None), "mm_save")


def binary_size(path):
    """(dims, value type) of an MCNLA dense binary file; dims[0] is the contiguous one."""
    dims = (ctypes.c_int64 * 3)()
    nd = ctypes.c_int()
    vt = ctypes.create_string_buffer(9)
    _lib.check(_lib.load().mcnla_b200_binary_size(_path(path), dims, ctypes.byref(nd), vt), "binary_size")
    return tuple(int(dims[i]) for i in range(nd.value)), vt.value.decode()


def load_binary(path, first=0, count=None):
    """Slices [first, first + count) along the last dimension as a float64 C-order array
    of shape (count, dims[-2], ..., dims[0]): rows of the reference's row-major matrix
    (dims {n, m}), columns of a column-major one (dims {m, n})."""
    dims, _ = binary_size(path)
    if count is None:
        count = dims[-1] - first
    out = np.empty((count,) + tuple(reversed(dims[:-1])), dtype=np.float64)
    _lib.check(_lib.load().mcnla_b200_binary_load(_path(path), first, count, out.ctypes.data_as(ctypes.c_void_p)),
               "binary_load")
    return out


def save_binary(path, a, comment=None):
    """Writes a C-order array as an R8 dense binary file, dims = reversed shape (a row-major
    m x n matrix gets dims {n, m}, as the reference writes its row-major matrices)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    dims = (ctypes.c_int64 * a.ndim)(*reversed(a.shape))
    _lib.check(_lib.load().mcnla_b200_binary_save(_path(path), a.ctypes.data_as(ctypes.c_void_p), a.ndim, dims,
                                                  comment.encode() if comment else None), "binary_save")


def binary_row_reader(path):
    """(m, n, read_rows) for a row-major MCNLA dense binary matrix file (dims {n, m}):
    read_rows(row0, rows, buf) loads rows [row0, row0 + rows) straight into the float64 buffer
    at address buf (the reference's loadBinaryRowBlock), for isvd.solve_stream."""
    dims, _ = binary_size(path)
    if len(dims) != 2:
        raise ValueError("%s: not a matrix" % path)
    n, m = dims
    lib = _lib.load()
    p = _path(path)

    def read_rows(row0, rows, buf):
        _lib.check(lib.mcnla_b200_binary_load(p, int(row0), int(rows), ctypes.c_void_p(buf)), "binary_load")
    return m, n, read_rows


def to_device(a, device="cuda"):
    """A host matrix on the device as float64, staged through pinned memory; a column-major
    array stays column-major (the transposed view of a row-major device tensor)."""
    import torch
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 2 and a.flags.f_contiguous and not a.flags.c_contiguous:
        return torch.from_numpy(a.T).pin_memory().to(device, non_blocking=True).t()
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(device, non_blocking=True)
