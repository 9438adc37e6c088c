"""CPU checks of the row-block decomposition's host side (no GPU): the row split, the
callback type the C ABI declares, and the torch.distributed all-reduce callback on two
gloo ranks (host buffers)."""
import ctypes
import os
import re
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mcnla_b200 import _lib, rowblock

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("m,world", [(1000, 2), (1001, 2), (7, 3), (3, 4), (100000, 8)])
def test_row_range_partitions_the_rows(m, world):
    blocks = [rowblock.row_range(m, world, r) for r in range(world)]
    assert blocks[0][0] == 0 and blocks[-1][1] == m
    for (a0, a1), (b0, b1) in zip(blocks, blocks[1:]):
        assert a1 == b0
    sizes = [b - a for a, b in blocks]
    assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_callback_type_matches_the_header():
    text = open(_lib.HEADER_PATH).read()
    assert re.search(r"typedef int \(\*mcnla_b200_allreduce_fn\)\(void\* user, double\* buf, int64_t count, "
                     r"void\* stream\);", text)
    assert _lib.ALLREDUCE_FN._restype_ is ctypes.c_int
    assert _lib.ALLREDUCE_FN._argtypes_ == (ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p)
    assert "#define MCNLA_B200_NCCL_ID_BYTES 128" in text and _lib.NCCL_ID_BYTES == 128


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ranks(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    from mcnla_b200 import rowblock as rb
    cb = rb.TorchAllReduce("cpu")
    x = np.arange(10, dtype=np.float64) * (rank + 1)
    fn = cb.cfn                          # called through the C function pointer, as the library does
    rc = fn(None, x.ctypes.data, 10, None)
    out[rank] = (rc, x.tolist(), cb.calls)
    dist.destroy_process_group()


def test_torch_allreduce_callback_two_gloo_ranks():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_ranks, args=(2, port, out), nprocs=2, join=True)
        want = (np.arange(10) * 3.0).tolist()
        assert dict(out) == {0: (0, want, 1), 1: (0, want, 1)}
