"""Python mirror of MCNLA's ``mcnla::isvd`` stage API on the B200 kernels.

The classes keep the reference's names, constructor arguments, setters and
getters (include/mcnla/isvd/**), so a test or driver reads like the
reference's own (check/isvd/**.cpp, src/isvd_dense_rb.cpp):

    params = Parameters().setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N).sync()
    sketcher = GaussianProjectionSketcher(params, seed); sketcher.initialize()
    ...
    q = params.createCollectionQ(); sketcher(a, q)

Every matrix is a CUDA float64 torch tensor (torch only provides device memory
and the stream); the work runs in ``libmcnla_b200.so`` through its C ABI.
Row-major means a C-contiguous tensor; a column-major m x n matrix is the
transpose view of a contiguous n x m tensor (strides (1, m)).

Differences from the reference, by design of the one-GPU build:
  * MPI arguments are accepted and ignored (one rank; sketches and row blocks
    are batched on the device).
  * The sketchers draw Omega on the device (Philox + Box-Muller) from the seed;
    ``setOmega`` passes Omega explicitly instead (the reference's stream depends
    on its thread count and cannot be reproduced bit for bit).
"""
import ctypes

import torch

from . import _lib

__all__ = [
    "Parameters", "Context", "context",
    "GaussianProjectionSketcher", "RowBlockGaussianProjectionSketcher", "ColBlockGaussianProjectionSketcher",
    "GramianOrthogonalizer", "RowBlockGramianOrthogonalizer",
    "KolmogorovNagumoIntegrator", "RowBlockKolmogorovNagumoIntegrator", "RowBlockGramianKolmogorovNagumoIntegrator",
    "RowBlockWenYinIntegrator", "RowBlockGramianWenYinIntegrator",
    "SvdFormer", "GramianFormer", "RowBlockGramianFormer", "ColBlockGramianFormer",
    "solve", "solve_host", "solve_stream", "Split", "split_bf16", "gaussian_bf16", "gemm_bf16", "solve_mixed",
    "Request", "Server", "solve_batched", "solve_grouped", "grouped_times", "resident_parts",
]


# ----------------------------------------------------------------------------------------------
# context
# ----------------------------------------------------------------------------------------------
class Context:
    """One ``mcnla_b200_ctx`` per device, bound to torch's current stream on every call."""

    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("mcnla_b200 needs a CUDA device (no CPU fallback)")
        self.lib = _lib.load()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self.lib.mcnla_b200_create(ctypes.byref(h), self.device.index, ctypes.c_void_p(stream)),
                   "mcnla_b200_create")
        self.handle = h
        self._stream = stream

    def bind(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        if s != self._stream:
            _lib.check(self.lib.mcnla_b200_set_stream(self.handle, ctypes.c_void_p(s)), "mcnla_b200_set_stream")
            self._stream = s
        return self.handle

    def last_times(self):
        buf = (ctypes.c_double * 16)()
        n = self.lib.mcnla_b200_last_times(self.handle, buf, 16)
        if n < 0:
            _lib.check(-n, "mcnla_b200_last_times")
        return [buf[i] for i in range(n)]

    def kernels_launched(self):
        return int(self.lib.mcnla_b200_kernels_launched(self.handle))

    def graph_replays(self):
        return int(self.lib.mcnla_b200_graph_replays(self.handle))

    def set_autotune(self, on):
        """GEMM tile autotuner on (default) or off (fixed shape heuristic)."""
        _lib.check(self.lib.mcnla_b200_set_autotune(self.handle, 1 if on else 0), "set_autotune")

    def set_cta_limit(self, ctas):
        """At most `ctas` CTAs for the persistent integrator kernels (0: one per SM)."""
        _lib.check(self.lib.mcnla_b200_set_cta_limit(self.handle, int(ctas)), "set_cta_limit")

    def set_graph_loop(self, on):
        """KN iteration loops as replayed CUDA graphs (default on) or direct launches."""
        _lib.check(self.lib.mcnla_b200_set_graph_loop(self.handle, 1 if on else 0), "set_graph_loop")

    def set_kn_method(self, method):
        """_lib.KN_AUTO (matrix functions, eigen fallback) or _lib.KN_EIGEN."""
        _lib.check(self.lib.mcnla_b200_set_kn_method(self.handle, method), "set_kn_method")

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mcnla_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts = {}


def context(device=None):
    dev = torch.cuda.current_device() if device is None else torch.device(device).index
    if dev not in _contexts:
        _contexts[dev] = Context(dev)
    return _contexts[dev]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _check_dev(t, name, shape=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64:
        raise TypeError("%s must be a CUDA float64 tensor" % name)
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError("%s has shape %s, expected %s" % (name, tuple(t.shape), tuple(shape)))


def _layout(a, name="A"):
    """(layout, lda) of a row-major (contiguous) or column-major (transposed contiguous) matrix."""
    if a.dim() != 2:
        raise ValueError("%s must be a matrix" % name)
    m, n = a.shape
    if a.stride(1) == 1 and a.stride(0) >= max(n, 1):
        return _lib.ROW_MAJOR, a.stride(0)
    if a.stride(0) == 1 and a.stride(1) >= max(m, 1):
        return _lib.COL_MAJOR, a.stride(1)
    raise ValueError("%s must be row-major or column-major with unit stride" % name)


def _rowmajor(t, name):
    if not t.is_contiguous():
        raise ValueError("%s must be row-major (C-contiguous)" % name)


# ----------------------------------------------------------------------------------------------
# Parameters (include/mcnla/isvd/core/parameters.hh:31-119)
# ----------------------------------------------------------------------------------------------
class Parameters:
    def __init__(self, mpi_root=0, mpi_comm=None, device=None):
        self.mpi_comm = mpi_comm
        self.mpi_size = 1
        self.mpi_root = mpi_root
        self.mpi_rank = 0
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None and \
            torch.cuda.is_available() else (torch.device(device) if device is not None else None)
        self._nrow = 0
        self._ncol = 0
        self._rank = 0
        self._over_rank = 12     # parameters.hh:63
        self._num_sketch = 16    # parameters.hh:66
        self._synchronized = False

    # setters (parameters.hpp:205-283) return self for chaining
    def setSize(self, nrow, ncol=None):
        if ncol is None:
            nrow, ncol = nrow.shape
        if nrow <= 0 or ncol <= 0:
            raise ValueError("sizes must be positive")
        self._nrow, self._ncol = int(nrow), int(ncol)
        self._synchronized = False
        return self

    def setRank(self, rank):
        if rank <= 0:
            raise ValueError("rank must be positive")
        self._rank = int(rank)
        self._synchronized = False
        return self

    def setOverRank(self, over_rank):
        if over_rank < 0:
            raise ValueError("over rank must be non-negative")
        self._over_rank = int(over_rank)
        self._synchronized = False
        return self

    def setNumSketch(self, num_sketch):
        if num_sketch <= 0:
            raise ValueError("number of sketches must be positive")
        self._num_sketch = int(num_sketch)
        self._synchronized = False
        return self

    def setNumSketchEach(self, num_sketch_each):
        return self.setNumSketch(num_sketch_each * self.mpi_size)

    def sync(self):
        # parameters.hpp:40-46 (the broadcast is a no-op with one rank)
        if self._nrow <= 0 or self._ncol <= 0 or self._rank <= 0:
            raise ValueError("set the size and the rank before sync()")
        if self.dimSketch() > _lib.MAX_DIM_SKETCH:
            raise ValueError("dimSketch %d exceeds %d" % (self.dimSketch(), _lib.MAX_DIM_SKETCH))
        self._synchronized = True
        return self

    # getters (parameters.hpp:53-197)
    def isSynchronized(self): return self._synchronized
    def nrow(self): return self._nrow
    def ncol(self): return self._ncol
    def nrowRank(self): return self._nrow
    def ncolRank(self): return self._ncol
    def nrowEach(self): return self._nrow
    def ncolEach(self): return self._ncol
    def nrowTotal(self): return self._nrow
    def ncolTotal(self): return self._ncol
    def rowrange(self): return (0, self._nrow)
    def colrange(self): return (0, self._ncol)
    def rank(self): return self._rank
    def overRank(self): return self._over_rank
    def dimSketch(self): return self._rank + self._over_rank
    def dimSketchEach(self): return self.dimSketch() * self.numSketchEach()
    def dimSketchTotal(self): return self.dimSketch() * self._num_sketch
    def numSketch(self): return self._num_sketch
    def numSketchEach(self): return self._num_sketch // self.mpi_size

    def c_params(self):
        return _lib.Params(self._nrow, self._ncol, self._rank, self._over_rank, self._num_sketch)

    # factories (parameters.hpp:288-363)
    def _empty(self, *shape):
        return torch.empty(*shape, dtype=torch.float64, device=self.device)

    def createCollectionQ(self): return self._empty(self._nrow, self.dimSketchTotal())
    createCollectionQj = createCollectionQ
    createCollectionQjp = createCollectionQ
    def createMatrixQbar(self): return self._empty(self._nrow, self.dimSketch())
    createMatrixQbarj = createMatrixQbar
    def createMatrixU(self): return self._empty(self._nrow, self._rank)
    createMatrixUj = createMatrixU
    def createMatrixV(self): return self._empty(self._ncol, self._rank)
    createMatrixVj = createMatrixV


# ----------------------------------------------------------------------------------------------
# StageWrapper (include/mcnla/isvd/core/stage_wrapper.hh:35-101)
# ----------------------------------------------------------------------------------------------
class _Stage:
    name_ = ""
    names_ = ""

    def __init__(self, parameters):
        self.parameters_ = parameters
        self.initialized_ = False
        self.computed_ = False
        self.moments_ = []

    def initialize(self):
        if not self.parameters_.isSynchronized():
            raise RuntimeError("parameters are not synchronized")
        self._initializeImpl()
        self.moments_ = []
        self.initialized_ = True
        self.computed_ = False

    def _initializeImpl(self):
        ctx = context(self.parameters_.device)
        p = self.parameters_.c_params()
        _lib.check(ctx.lib.mcnla_b200_initialize(ctx.bind(), ctypes.byref(p), -1, -1), "initialize")

    def __call__(self, *args):
        if not self.parameters_.isSynchronized():
            raise RuntimeError("parameters are not synchronized")
        if not self.initialized_:
            raise RuntimeError("stage is not initialized")
        self.moments_ = []
        self._runImpl(*args)
        self.computed_ = True
        return self

    def _record_times(self, ctx):
        times = ctx.last_times()
        t = 0.0
        self.moments_ = [0.0]
        for x in times:
            t += x
            self.moments_.append(t)

    def isInitialized(self): return self.initialized_
    def isComputed(self): return self.computed_

    def time(self):
        return self.moments_[-1] - self.moments_[0] if self.moments_ else 0.0

    def times(self):
        if not self.computed_:
            raise RuntimeError("stage is not computed")
        return [b - a for a, b in zip(self.moments_[:-1], self.moments_[1:])]

    def moments(self): return list(self.moments_)
    def commTime(self): return 0.0
    def commTimes(self): return [0.0] * max(len(self.moments_) - 1, 0)
    def names(self): return self.names_
    def __str__(self): return self.name_


# ----------------------------------------------------------------------------------------------
# Sketchers (include/mcnla/isvd/sketcher/)
# ----------------------------------------------------------------------------------------------
class GaussianProjectionSketcher(_Stage):
    name_ = "Gaussian Projection Sketcher"
    names_ = "random generating / projection"
    _max_exponent = None

    def __init__(self, parameters, seed=0, exponent=0):
        super().__init__(parameters)
        self._omega_given = None
        self.setSeed(seed)
        self.setExponent(exponent)

    def seed(self): return self.seed_
    def exponent(self): return self.exponent_

    def setSeed(self, seed):
        self.seed_ = int(seed)
        self.computed_ = False
        return self

    def setExponent(self, exponent):
        if exponent < 0 or (self._max_exponent is not None and exponent > self._max_exponent):
            raise ValueError("invalid exponent for %s" % self.name_)
        self.exponent_ = int(exponent)
        self.computed_ = False
        return self

    def setOmega(self, omega):
        """Uses the given n x (N*l) row-major Omega instead of drawing one."""
        self._omega_given = omega
        self.computed_ = False
        return self

    def matrixOmega(self):
        return self.omega_

    def _runImpl(self, matrix_a, collection_q):
        p = self.parameters_
        m, n, L = p.nrow(), p.ncol(), p.dimSketchTotal()
        _check_dev(matrix_a, "A", (m, n))
        _check_dev(collection_q, "Q", (m, L))
        _rowmajor(collection_q, "Q")
        layout, lda = _layout(matrix_a)
        ctx = context(p.device)
        h = ctx.bind()
        if self._omega_given is not None:
            _check_dev(self._omega_given, "Omega", (n, L))
            om = self._omega_given.contiguous()
            if self.exponent_ > 0:
                om = om.clone()
        else:
            om = torch.empty(n, L, dtype=torch.float64, device=matrix_a.device)
            _lib.check(ctx.lib.mcnla_b200_gaussian(h, ctypes.c_uint64(self.seed_ & (2**64 - 1)), n * L, _ptr(om)),
                       "gaussian")
        self.omega_ = om
        cp = p.c_params()
        _lib.check(ctx.lib.mcnla_b200_sketch(h, ctypes.byref(cp), _ptr(matrix_a), layout, lda, _ptr(om),
                                             self.exponent_, _ptr(collection_q)), "sketch")
        self._record_times(ctx)


class RowBlockGaussianProjectionSketcher(GaussianProjectionSketcher):
    name_ = "Gaussian Projection Sketcher (Row-Block Version)"
    _max_exponent = 0   # row_block_gaussian_projection_sketcher.hpp:160-168


class ColBlockGaussianProjectionSketcher(GaussianProjectionSketcher):
    name_ = "Gaussian Projection Sketcher (Column-Block Version)"
    _max_exponent = 0

    def __init__(self, parameters, seed=0):
        super().__init__(parameters, seed, 0)


# ----------------------------------------------------------------------------------------------
# Orthogonalizers (include/mcnla/isvd/orthogonalizer/)
# ----------------------------------------------------------------------------------------------
class GramianOrthogonalizer(_Stage):
    name_ = "Gramian Orthogonalizer"
    names_ = "orthogonalization"

    def _runImpl(self, collection_q):
        p = self.parameters_
        _check_dev(collection_q, "Q", (p.nrow(), p.dimSketchTotal()))
        _rowmajor(collection_q, "Q")
        ctx = context(p.device)
        cp = p.c_params()
        _lib.check(ctx.lib.mcnla_b200_orthogonalize(ctx.bind(), ctypes.byref(cp), _ptr(collection_q)),
                   "orthogonalize")
        self._record_times(ctx)


class RowBlockGramianOrthogonalizer(GramianOrthogonalizer):
    name_ = "Gramian Orthogonalizer (Row-Block Version)"


# ----------------------------------------------------------------------------------------------
# Integrators (include/mcnla/isvd/integrator/)
# ----------------------------------------------------------------------------------------------
class _Integrator(_Stage):
    _kind = None
    _default_tol = 1e-4

    def __init__(self, parameters, max_iteration=256, tolerance=None):
        super().__init__(parameters)
        self.setMaxIteration(max_iteration)
        self.setTolerance(self._default_tol if tolerance is None else tolerance)
        self.iteration_ = 0

    def maxIteration(self): return self.max_iteration_
    def tolerance(self): return self.tolerance_

    def iteration(self):
        if not self.computed_:
            raise RuntimeError("stage is not computed")
        return self.iteration_

    def setMaxIteration(self, max_iteration):
        if max_iteration < 0:
            raise ValueError("max iteration must be non-negative")
        self.max_iteration_ = int(max_iteration)
        self.initialized_ = False
        self.computed_ = False
        return self

    def setTolerance(self, tolerance):
        if not tolerance >= 0:
            raise ValueError("tolerance must be non-negative")
        self.tolerance_ = float(tolerance)
        self.initialized_ = False
        self.computed_ = False
        return self

    def _runImpl(self, collection_q, matrix_qbar):
        p = self.parameters_
        _check_dev(collection_q, "Q", (p.nrow(), p.dimSketchTotal()))
        _check_dev(matrix_qbar, "Qbar", (p.nrow(), p.dimSketch()))
        _rowmajor(collection_q, "Q")
        _rowmajor(matrix_qbar, "Qbar")
        ctx = context(p.device)
        cp = p.c_params()
        it = ctypes.c_int()
        _lib.check(ctx.lib.mcnla_b200_integrate(ctx.bind(), ctypes.byref(cp), self._kind, _ptr(collection_q),
                                                self.max_iteration_, self.tolerance_, _ptr(matrix_qbar),
                                                ctypes.byref(it)), "integrate")
        self.iteration_ = it.value
        self._record_times(ctx)


class KolmogorovNagumoIntegrator(_Integrator):
    name_ = "Kolmogorov-Nagumo-Type Integrator"
    names_ = "copying Qc / iterating"
    _kind = _lib.KOLMOGOROV_NAGUMO


class RowBlockKolmogorovNagumoIntegrator(_Integrator):
    name_ = "Kolmogorov-Nagumo-Type Integrator (Row-Block Version)"
    names_ = "initializing / iterating"
    _kind = _lib.ROW_BLOCK_KOLMOGOROV_NAGUMO


class RowBlockGramianKolmogorovNagumoIntegrator(_Integrator):
    name_ = "Kolmogorov-Nagumo-Type Integrator (Row-Block Gramian Version)"
    names_ = "initializing / iterating / forming Qbar"
    _kind = _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO


class RowBlockWenYinIntegrator(_Integrator):
    name_ = "Wen-Yin Line Search Integrator (Row-Block Version)"
    names_ = "initializing / iterating"
    _kind = _lib.ROW_BLOCK_WEN_YIN
    _default_tol = 1e-3


class RowBlockGramianWenYinIntegrator(_Integrator):
    name_ = "Wen-Yin Line Search Integrator (Row-Block Gramian Version)"
    names_ = "initializing / iterating / forming Qbar"
    _kind = _lib.ROW_BLOCK_GRAMIAN_WEN_YIN
    _default_tol = 1e-3


# ----------------------------------------------------------------------------------------------
# Formers (include/mcnla/isvd/former/)
# ----------------------------------------------------------------------------------------------
class _Former(_Stage):
    _kind = None

    def __init__(self, parameters, jobv=True):
        super().__init__(parameters)
        self.jobv_ = bool(jobv)
        self.s_ = self.u_ = self.v_ = None

    def _runImpl(self, matrix_a, matrix_qbar):
        p = self.parameters_
        m, n, k = p.nrow(), p.ncol(), p.rank()
        _check_dev(matrix_a, "A", (m, n))
        _check_dev(matrix_qbar, "Qbar", (m, p.dimSketch()))
        _rowmajor(matrix_qbar, "Qbar")
        layout, lda = _layout(matrix_a)
        dev = matrix_a.device
        self.s_ = torch.empty(k, dtype=torch.float64, device=dev)
        self.u_ = torch.empty(m, k, dtype=torch.float64, device=dev)
        self.v_ = torch.empty(n, k, dtype=torch.float64, device=dev) if self.jobv_ else None
        ctx = context(p.device)
        cp = p.c_params()
        _lib.check(ctx.lib.mcnla_b200_form(ctx.bind(), ctypes.byref(cp), self._kind, _ptr(matrix_a), layout, lda,
                                           _ptr(matrix_qbar), _ptr(self.s_), _ptr(self.u_), _ptr(self.v_)), "form")
        self._record_times(ctx)

    def vectorS(self):
        self._need()
        return self.s_

    def matrixU(self):
        self._need()
        return self.u_

    def matrixV(self):
        self._need()
        if not self.jobv_:
            raise RuntimeError("V was not requested")
        return self.v_

    def _need(self):
        if not self.computed_:
            raise RuntimeError("stage is not computed")


class SvdFormer(_Former):
    names_ = "Projection / SVD / forming"
    _kind = _lib.SVD_FORMER

    @property
    def name_(self):
        return "SVD Former" if self.jobv_ else "SVD Former (without V)"


class GramianFormer(_Former):
    names_ = "Projection / eigen / forming"
    _kind = _lib.GRAMIAN_FORMER

    @property
    def name_(self):
        return "Gramian Former" if self.jobv_ else "Gramian Former (without V)"


class RowBlockGramianFormer(_Former):
    names_ = "Projection / eigen / forming"
    _kind = _lib.ROW_BLOCK_GRAMIAN_FORMER
    name_ = "Gramian Former (Row-Block Version)"

    def matrixUj(self): return self.matrixU()
    def matrixVj(self): return self.matrixV()


class ColBlockGramianFormer(_Former):
    names_ = "Projection / eigen / forming"
    _kind = _lib.COL_BLOCK_GRAMIAN_FORMER
    name_ = "Gramian Former (Column-Block Version)"

    def matrixVj(self): return self.matrixV()


# ----------------------------------------------------------------------------------------------
# Whole solves (the drivers' wiring, src/isvd_dense_rb.cpp:46-286)
# ----------------------------------------------------------------------------------------------
INTEGRATORS = {
    "kn": _lib.KOLMOGOROV_NAGUMO, "rb_kn": _lib.ROW_BLOCK_KOLMOGOROV_NAGUMO,
    "rb_gramian_kn": _lib.ROW_BLOCK_GRAMIAN_KOLMOGOROV_NAGUMO, "rb_wy": _lib.ROW_BLOCK_WEN_YIN,
    "rb_gramian_wy": _lib.ROW_BLOCK_GRAMIAN_WEN_YIN,
}
FORMERS = {"svd": _lib.SVD_FORMER, "gramian": _lib.GRAMIAN_FORMER, "rb_gramian": _lib.ROW_BLOCK_GRAMIAN_FORMER,
           "cb_gramian": _lib.COL_BLOCK_GRAMIAN_FORMER}


def solve(a, k, p, N, omega=None, seed=0, integrator="kn", former="svd", maxit=256, tol=1e-4, with_v=True):
    """One whole iSVD on device buffers through ``mcnla_b200_isvd``.  Returns (S, U, V, iterations)."""
    m, n = a.shape
    _check_dev(a, "A")
    layout, lda = _layout(a)
    prm = _lib.Params(m, n, k, p, N)
    dev = a.device
    s = torch.empty(k, dtype=torch.float64, device=dev)
    u = torch.empty(m, k, dtype=torch.float64, device=dev)
    v = torch.empty(n, k, dtype=torch.float64, device=dev) if with_v else None
    if omega is not None:
        _check_dev(omega, "Omega", (n, (k + p) * N))
        omega = omega.contiguous()
    ctx = context(dev)
    it = ctypes.c_int()
    _lib.check(ctx.lib.mcnla_b200_isvd(ctx.bind(), ctypes.byref(prm), INTEGRATORS[integrator], FORMERS[former],
                                       _ptr(a), layout, lda, _ptr(omega), ctypes.c_uint64(seed), maxit, tol, _ptr(s),
                                       _ptr(u), _ptr(v), ctypes.byref(it)), "isvd")
    return s, u, v, it.value


def solve_host(a_host, omega_host, k, p, N, integrator="kn", former="svd", maxit=256, tol=1e-4, out=None,
               colmajor=False, device=None):
    """One whole iSVD from HOST buffers through ``mcnla_b200_isvd_host`` (copies in and out
    inside the call).  a_host: CPU float64 tensor m x n (row-major; or its column-major
    buffer when colmajor); omega_host: CPU float64 n x (N*l).  Returns (S, U, V, iterations)
    as CPU tensors (the ``out`` triple is reused when given)."""
    if colmajor:
        n, m = a_host.shape
    else:
        m, n = a_host.shape
    for t, name in ((a_host, "A"), (omega_host, "Omega")):
        if t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
            raise TypeError("%s must be a contiguous CPU float64 tensor" % name)
    if out is None:
        pin = a_host.is_pinned()
        out = (torch.empty(k, dtype=torch.float64, pin_memory=pin),
               torch.empty(m, k, dtype=torch.float64, pin_memory=pin),
               torch.empty(n, k, dtype=torch.float64, pin_memory=pin))
    s, u, v = out
    prm = _lib.Params(m, n, k, p, N)
    ctx = context(device)
    it = ctypes.c_int()
    _lib.check(ctx.lib.mcnla_b200_isvd_host(ctx.bind(), ctypes.byref(prm), INTEGRATORS[integrator], FORMERS[former],
                                            _ptr(a_host), _lib.COL_MAJOR if colmajor else _lib.ROW_MAJOR,
                                            _ptr(omega_host), maxit, tol, _ptr(s), _ptr(u), _ptr(v),
                                            ctypes.byref(it)), "isvd_host")
    return s, u, v, it.value


def solve_stream(read_rows, m, n, omega_host, k, p, N, integrator="kn", former="svd", maxit=256, tol=1e-4,
                 out=None, device=None):
    """One whole iSVD of a row-major m x n A that ``read_rows(row0, rows, buf)`` produces block by
    block (``buf``: the address of a pinned rows x n float64 buffer to fill; e.g.
    io.binary_row_reader(path)), through ``mcnla_b200_isvd_stream``: each block is copied and
    sketched on the device while the next one is read.  omega_host: CPU float64 n x (N*l).
    Returns (S, U, V, iterations) as CPU tensors, bit-identical to solve_host on the same A."""
    if omega_host.is_cuda or omega_host.dtype != torch.float64 or not omega_host.is_contiguous():
        raise TypeError("Omega must be a contiguous CPU float64 tensor")
    if out is None:
        out = (torch.empty(k, dtype=torch.float64, pin_memory=True),
               torch.empty(m, k, dtype=torch.float64, pin_memory=True),
               torch.empty(n, k, dtype=torch.float64, pin_memory=True))
    s, u, v = out
    failure = []

    def call(_user, row0, rows, buf):
        try:
            read_rows(int(row0), int(rows), int(buf))
            return 0
        except Exception as e:            # reported by the library as a reader error
            failure.append(e)
            return 1
    cb = _lib.READ_ROWS_FN(call)
    prm = _lib.Params(m, n, k, p, N)
    ctx = context(device)
    it = ctypes.c_int()
    st = ctx.lib.mcnla_b200_isvd_stream(ctx.bind(), ctypes.byref(prm), INTEGRATORS[integrator], FORMERS[former], cb,
                                        None, _ptr(omega_host), maxit, tol, _ptr(s), _ptr(u), _ptr(v),
                                        ctypes.byref(it))
    if failure:
        raise failure[0]
    _lib.check(st, "isvd_stream")
    return s, u, v, it.value


# ----------------------------------------------------------------------------------------------
# Mixed precision: BF16 tensor-core sketch (tcgen05), FP64 elsewhere
# ----------------------------------------------------------------------------------------------
def _bf16_buffer(rows, cols, dev):
    """rows x cols BF16 with a row pitch that is a multiple of 8 elements (16 bytes)."""
    ld = (cols + 7) // 8 * 8
    buf = torch.zeros(rows, ld, dtype=torch.bfloat16, device=dev)
    return buf[:, :cols], ld


class Split(tuple):
    """BF16 parts of A: (hi, lo, lo2, pitch); lo / lo2 are None when not split out."""
    __slots__ = ()

    def __new__(cls, hi, lo, lo2, ld):
        return tuple.__new__(cls, (hi, lo, lo2, ld))

    hi = property(lambda self: self[0])
    lo = property(lambda self: self[1])
    lo2 = property(lambda self: self[2])
    ld = property(lambda self: self[3])

    @property
    def parts(self):
        return 1 + (self[1] is not None) + (self[2] is not None)


def split_bf16(a, parts=2):
    """A = A_hi + A_lo (+ A_lo2) in BF16 (row-major views with 16-byte pitch), parts in 1..3:
    8, 16 or 24 bits of mantissa (three parts hold an FP32 A exactly).  Returns a Split."""
    if parts not in (1, 2, 3):
        raise ValueError("parts must be 1, 2 or 3")
    _check_dev(a, "A")
    layout, lda = _layout(a)
    m, n = a.shape
    hi, ld = _bf16_buffer(m, n, a.device)
    lo = _bf16_buffer(m, n, a.device)[0] if parts >= 2 else None
    lo2 = _bf16_buffer(m, n, a.device)[0] if parts >= 3 else None
    ctx = context(a.device)
    _lib.check(ctx.lib.mcnla_b200_split_bf16(ctx.bind(), _ptr(a), layout, lda, m, n, _ptr(hi), _ptr(lo), _ptr(lo2),
                                             ld), "split_bf16")
    return Split(hi, lo, lo2, ld)


def resident_parts(a, parts=3):
    """The BF16 parts a served matrix keeps resident (split once, not per request): `parts` parts of A
    for the mixed sketch and three of A' for the precision former, as (Split, Split).  A may be FP32
    or FP64 (an FP32 A is widened for the split only; its parts are those of the exact FP64 copy)."""
    a64 = a if a.dtype == torch.float64 else a.double()
    out = split_bf16(a64, parts), split_bf16(a64.t(), 3)
    del a64
    return out


def gaussian_bf16(n, L, seed, device=None, with_fp64=False):
    """Omega' (L x n BF16, pitch multiple of 8) and optionally the same values as an n x L FP64 Omega."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    omega_t, ld = _bf16_buffer(L, n, dev)
    omega = torch.empty(n, L, dtype=torch.float64, device=dev) if with_fp64 else None
    ctx = context(dev)
    _lib.check(ctx.lib.mcnla_b200_gaussian_bf16(ctx.bind(), ctypes.c_uint64(seed), n, L, _ptr(omega_t), ld,
                                                _ptr(omega)), "gaussian_bf16")
    return omega_t, ld, omega


def gemm_bf16(a_hi, a_lo, lda, b, ldb, out_dtype=torch.float64, a_lo2=None):
    """D = (A_hi + A_lo + A_lo2) B' on tcgen05 (BF16 in, FP32 accumulation)."""
    M, K = a_hi.shape
    N = b.shape[0]
    d = torch.empty(M, N, dtype=out_dtype, device=a_hi.device)
    ctx = context(a_hi.device)
    _lib.check(ctx.lib.mcnla_b200_gemm_bf16(ctx.bind(), M, N, K, _ptr(a_hi), _ptr(a_lo), _ptr(a_lo2), lda, _ptr(b),
                                            ldb, _ptr(d), N, 1 if out_dtype == torch.float64 else 0), "gemm_bf16")
    return d


def form_bf16(at_split, qbar, k, p, N, former="svd", with_v=True):
    """Precision-form former: Q' A on tcgen05 from the BF16 parts of A' (`at_split`, e.g.
    split_bf16(a.t(), 3)) and a three-part split of Qbar, the rest in FP64.  Returns (S, U, V)."""
    at_hi, at_lo, at_lo2, ldt = at_split
    n, m = at_hi.shape[0], qbar.shape[0]
    _check_dev(qbar, "Qbar")
    if not qbar.is_contiguous():
        raise ValueError("Qbar must be a contiguous row-major m x l matrix")
    prm = _lib.Params(m, n, k, p, N)
    dev = qbar.device
    s = torch.empty(k, dtype=torch.float64, device=dev)
    u = torch.empty(m, k, dtype=torch.float64, device=dev)
    v = torch.empty(n, k, dtype=torch.float64, device=dev) if with_v else None
    ctx = context(dev)
    _lib.check(ctx.lib.mcnla_b200_form_bf16(ctx.bind(), ctypes.byref(prm), FORMERS[former], _ptr(at_hi), _ptr(at_lo),
                                            _ptr(at_lo2), ldt, _ptr(qbar), _ptr(s), _ptr(u), _ptr(v)), "form_bf16")
    return s, u, v


def solve_mixed(a, k, p, N, seed=0, integrator="kn", former="svd", maxit=256, tol=1e-4, split=None, with_v=True,
                parts=2, former_split=None):
    """Whole iSVD with the BF16 tensor-core sketch (Omega drawn in BF16 from seed), FP64
    orthogonalizer / integrator steps, and the former in FP64 from A or, when `former_split`
    (the BF16 parts of A', e.g. split_bf16(a.t(), 3)) is given, in the precision form.
    `split` (a Split) reuses a resident BF16 copy of A; otherwise A is split into `parts` BF16
    parts.  Returns (S, U, V, iterations)."""
    m, n = a.shape
    _check_dev(a, "A")
    layout, lda = _layout(a)
    if split is None:
        split = split_bf16(a, parts)
    hi, lo, lo2, ld16 = split
    at_hi, at_lo, at_lo2, ldt = former_split if former_split is not None else (None, None, None, 0)
    prm = _lib.Params(m, n, k, p, N)
    dev = a.device
    s = torch.empty(k, dtype=torch.float64, device=dev)
    u = torch.empty(m, k, dtype=torch.float64, device=dev)
    v = torch.empty(n, k, dtype=torch.float64, device=dev) if with_v else None
    ctx = context(dev)
    it = ctypes.c_int()
    _lib.check(ctx.lib.mcnla_b200_isvd_mixed(ctx.bind(), ctypes.byref(prm), INTEGRATORS[integrator], FORMERS[former],
                                             _ptr(a), layout, lda, _ptr(hi), _ptr(lo), _ptr(lo2), ld16,
                                             _ptr(at_hi), _ptr(at_lo), _ptr(at_lo2), ldt, ctypes.c_uint64(seed),
                                             maxit, tol, _ptr(s), _ptr(u), _ptr(v), ctypes.byref(it)), "isvd_mixed")
    return s, u, v, it.value


# ----------------------------------------------------------------------------------------------
# Batched and served solves (mcnla_b200_server_*)
# ----------------------------------------------------------------------------------------------
class Request:
    """One solve for the server: A (CUDA float64 or float32, row- or column-major) and its
    parameters; the outputs S, U, V are allocated here on A's device.  mixed: False (FP64),
    True or 2 (BF16 hi+lo sketch) or 3 (BF16 hi+lo+lo2 sketch); the mixed solves run the
    precision former from three BF16 parts of A'.  split / former_split: resident BF16 parts of
    A and of A' (split_bf16(a, parts), split_bf16(a.t(), 3)) kept by the caller; without them
    each solve splits A itself."""

    def __init__(self, a, k, p, N, seed=0, integrator="kn", former="svd", maxit=256, tol=1e-4, mixed=False,
                 with_v=True, split=None, former_split=None):
        if not isinstance(a, torch.Tensor) or not a.is_cuda or a.dtype not in (torch.float64, torch.float32):
            raise TypeError("A must be a CUDA float64 or float32 tensor")
        layout, lda = _layout(a)
        m, n = a.shape
        dev = a.device
        self.a = a
        self.s = torch.empty(k, dtype=torch.float64, device=dev)
        self.u = torch.empty(m, k, dtype=torch.float64, device=dev)
        self.v = torch.empty(n, k, dtype=torch.float64, device=dev) if with_v else None
        pr = _lib.Problem()
        pr.params = _lib.Params(m, n, k, p, N)
        pr.A = a.data_ptr() if a.dtype == torch.float64 else None
        pr.A32 = a.data_ptr() if a.dtype == torch.float32 else None
        pr.a_layout = layout
        pr.lda = lda
        pr.seed = seed
        pr.integrator = INTEGRATORS[integrator]
        pr.former = FORMERS[former]
        pr.max_iteration = maxit
        pr.tolerance = tol
        if mixed is False or mixed is None or mixed == 0:
            pr.precision = _lib.PRECISION_FP64
        elif mixed is True or mixed == 2:
            pr.precision = _lib.PRECISION_MIXED
        elif mixed == 3:
            pr.precision = _lib.PRECISION_MIXED3
        else:
            raise ValueError("mixed must be False, True, 2 or 3")
        pr.S = self.s.data_ptr()
        pr.U = self.u.data_ptr()
        pr.V = self.v.data_ptr() if self.v is not None else None
        # resident BF16 parts of A (sketch) and of A' (precision former), split once by the caller
        self._keep = (split, former_split)
        if split is not None:
            pr.a_hi, pr.a_lo = split.hi.data_ptr(), split.lo.data_ptr()
            pr.a_lo2 = split.lo2.data_ptr() if split.lo2 is not None else None
            pr.lda16 = split.ld
        if former_split is not None:
            pr.at_hi, pr.at_lo, pr.at_lo2 = (t.data_ptr() for t in former_split[:3])
            pr.ldat16 = former_split.ld
        self.problem = pr
        self.ticket = None
        self.result = None

    def bytes(self):
        return int(_lib.load().mcnla_b200_problem_bytes(ctypes.byref(self.problem)))


class Server:
    """A pool of `workers` concurrent solvers on one device with an HBM admission budget."""

    def __init__(self, workers=4, budget_bytes=150 << 30, device=None):
        self.lib = _lib.load()
        dev = torch.cuda.current_device() if device is None else torch.device(device).index
        torch.cuda.synchronize(dev)
        h = ctypes.c_void_p()
        _lib.check(self.lib.mcnla_b200_server_create(ctypes.byref(h), dev, workers, budget_bytes), "server_create")
        self.handle = h

    def submit(self, req):
        t = ctypes.c_int64()
        _lib.check(self.lib.mcnla_b200_server_submit(self.handle, ctypes.byref(req.problem), ctypes.byref(t)),
                   "server_submit")
        req.ticket = t.value
        return req

    def wait(self, req):
        out = _lib.Problem()
        st = self.lib.mcnla_b200_server_wait(self.handle, req.ticket, ctypes.byref(out))
        req.result = out
        _lib.check(st, "server_wait")
        return req

    def stats(self):
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self.lib.mcnla_b200_server_stats(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                   "server_stats")
        return {"in_flight_bytes": a.value, "peak_bytes": b.value, "completed": c.value}

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mcnla_b200_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


BATCH_PHASES = ("sketch_orthogonalize_gramian", "grouped_kernel", "declined_iterations", "qbar_former",
                "other_problems", "kernel_bs_bc", "kernel_d_dg", "kernel_kn_step", "kernel_e_b_update")


def grouped_times():
    """Seconds of the phases of the last solve_grouped call (BATCH_PHASES order; the kernel_* entries are
    the grouped kernel's device time summed over the problems)."""
    buf = (ctypes.c_double * len(BATCH_PHASES))()
    _lib.load().mcnla_b200_grouped_times(buf, len(BATCH_PHASES))
    return dict(zip(BATCH_PHASES, (round(buf[i], 4) for i in range(len(BATCH_PHASES)))))


def _run_batch(entry, requests, workers, budget_bytes):
    if not requests:
        return requests
    torch.cuda.synchronize()
    arr = (_lib.Problem * len(requests))(*[r.problem for r in requests])
    dev = requests[0].a.device.index
    st = getattr(_lib.load(), entry)(dev, arr, len(requests), workers, budget_bytes)
    for r, out in zip(requests, arr):
        r.result = out
    _lib.check(st, entry)
    return requests


def solve_batched(requests, workers=4, budget_bytes=150 << 30):
    """All requests through one temporary worker pool (mcnla_b200_isvd_batched)."""
    return _run_batch("mcnla_b200_isvd_batched", requests, workers, budget_bytes)


def solve_grouped(requests, workers=4, budget_bytes=150 << 30):
    """All requests as a grouped batch (mcnla_b200_isvd_grouped): the row-block Gramian KN problems'
    iterations in one grouped kernel, the rest of every solve on `workers` workers."""
    return _run_batch("mcnla_b200_isvd_grouped", requests, workers, budget_bytes)
