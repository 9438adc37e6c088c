"""Row-block decomposition of one solve over several GPUs (one process per GPU).

The reference decomposes one iSVD over MPI ranks by rows of A
(src/isvd_dense_rb.cpp with the row-block stages): every rank holds a block of
rows, sketches it with the same Omega and keeps its rows of Q, Qbar and U; the
stages sum their row-dependent partial products over the ranks.  Here a
context gets a communicator (``attach_nccl``: the library's own NCCL
communicator over NVLink / NVSwitch; ``attach_torch``: an all-reduce through a
torch.distributed process group), after which every stage entry point and
``isvd.solve`` run on the rank's rows: pass the LOCAL row block of A as the
matrix; S, V and the iteration count come out the same on every rank, U holds
the rank's rows.  All ranks must make the same calls in the same order.
"""
import ctypes

import torch

from . import _lib
from . import isvd


def row_range(m, world, rank):
    """Rows [r0, r1) of rank `rank` when m rows are split over `world` ranks: the first
    m % world ranks take one row more (the reference's Parameters::rowrange split)."""
    if not (0 <= rank < world) or m < 0:
        raise ValueError("bad rank / world / m")
    base, extra = divmod(m, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


class _DeviceArray:
    """A view of `count` doubles at a device address, for torch.as_tensor."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None, "stream": None}


class TorchAllReduce:
    """mcnla_b200_allreduce_fn through torch.distributed.  With the NCCL backend the sum runs on
    the device, ordered after the work queued on the library's stream; with any other backend
    (gloo) the block is staged through host memory after a synchronization of that stream, which
    lets several ranks share one GPU in tests."""

    def __init__(self, device, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = torch.device(device)
        self.nccl = dist.get_backend(group) == "nccl"
        self.calls = 0
        self.error = None
        self.cfn = _lib.ALLREDUCE_FN(self._call)   # keep a reference: the library holds the pointer

    def _call(self, user, buf, count, stream):
        try:
            if self.device.type == "cpu":      # host buffers (the callback's own tests)
                import numpy as np
                arr = np.ctypeslib.as_array(ctypes.cast(buf, ctypes.POINTER(ctypes.c_double)), shape=(int(count),))
                self.dist.all_reduce(torch.from_numpy(arr), group=self.group)
                self.calls += 1
                return 0
            t = torch.as_tensor(_DeviceArray(buf, count), device=self.device)
            ext = torch.cuda.ExternalStream(int(stream), device=self.device) if stream else \
                torch.cuda.default_stream(self.device)
            with torch.cuda.stream(ext):
                if self.nccl:
                    self.dist.all_reduce(t, group=self.group)
                else:
                    ext.synchronize()
                    h = t.cpu()
                    self.dist.all_reduce(h, group=self.group)
                    t.copy_(h)
                    ext.synchronize()
            self.calls += 1
            return 0
        except Exception as e:  # reported to the library as a failed collective
            self.error = e
            return 1


def attach_torch(ctx, group=None):
    """Sums through torch.distributed (see TorchAllReduce).  Returns the callback object, which
    must stay alive while the context uses it."""
    cb = TorchAllReduce(ctx.device, group)
    _lib.check(ctx.lib.mcnla_b200_set_allreduce(ctx.bind(), cb.cfn, None), "set_allreduce")
    ctx._allreduce = cb
    return cb


def attach_nccl(ctx, rank=None, world=None, group=None):
    """The library's own NCCL communicator over the ranks of a torch.distributed group (its
    unique id is created on rank 0 and broadcast through the group; any backend)."""
    import torch.distributed as dist
    if world is None:
        world = dist.get_world_size(group) if dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank(group) if dist.is_initialized() else 0
    buf = ctypes.create_string_buffer(_lib.NCCL_ID_BYTES)
    if rank == 0:
        _lib.check(ctx.lib.mcnla_b200_nccl_unique_id(buf), "nccl_unique_id")
    if world > 1:
        obj = [buf.raw if rank == 0 else None]
        dist.broadcast_object_list(obj, src=0, group=group)
        ctypes.memmove(buf, obj[0], _lib.NCCL_ID_BYTES)
    _lib.check(ctx.lib.mcnla_b200_set_nccl(ctx.bind(), buf, world, rank), "set_nccl")


def detach(ctx):
    _lib.check(ctx.lib.mcnla_b200_set_allreduce(ctx.bind(), _lib.ALLREDUCE_FN(), None), "set_allreduce")
    ctx._allreduce = None


def allreduces(ctx):
    return ctx.lib.mcnla_b200_allreduces(ctx.bind())


def solve_row_block(a_local, k, p, N, omega=None, seed=0, integrator="rb_gramian_kn", former="rb_gramian",
                    maxit=256, tol=1e-4, with_v=True):
    """One iSVD of the matrix whose rows are split over the ranks: a_local is this rank's row
    block (device, FP64).  The context of a_local's device must have a communicator
    (attach_nccl / attach_torch).  Returns (S, U rows of this rank, V, iterations)."""
    return isvd.solve(a_local, k, p, N, omega=omega, seed=seed, integrator=integrator, former=former, maxit=maxit,
                      tol=tol, with_v=with_v)
