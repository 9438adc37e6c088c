"""GPU checks of the row-block decomposition of one solve (rows of A over ranks).

Two or three ranks share the one GPU of the test machine: each is its own process
with its own context, and their sums go through torch.distributed's gloo backend,
staged through host memory by the library's all-reduce callback, so no kernel of
one rank ever waits on another rank's kernels (the host collective orders them).
Each rank holds its block of rows of the same A and the same Omega; the result must
match the single-GPU solve of the whole matrix: singular values to 1e-10 relative,
U (the ranks' row blocks stacked) and V to 1e-10 up to column sign, and identical
iteration counts.  The library's own NCCL communicator is checked with one rank (a
second GPU is not available to these tests).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import isvd_oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOL = 1e-10

CASES = [
    # m, n, k, p, N, integrator, former, tol, world
    (1000, 600, 10, 6, 8, "rb_gramian_kn", "rb_gramian", 1e-5, 2),
    (1001, 600, 10, 6, 8, "rb_kn", "svd", 1e-5, 2),
    (900, 700, 8, 4, 6, "rb_wy", "gramian", 1e-4, 2),
    (1000, 500, 10, 6, 8, "kn", "svd", 1e-5, 3),
    (997, 400, 6, 6, 4, "rb_gramian_wy", "rb_gramian", 1e-4, 2),
]


def _inputs(m, n, k, p, N):
    from mcnla_b200 import synthetic
    a = synthetic.lowrank_np(m, n, 1.0 / np.arange(1, min(m, n) + 1) ** 1.5, seed=m + n)
    omega = np.random.default_rng(m).standard_normal((n, (k + p) * N))
    return a, omega


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, case, out):
    import datetime
    import sys
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(0)
    from mcnla_b200 import isvd, rowblock
    m, n, k, p, N, integ, former, tol, _ = case
    a, omega = _inputs(m, n, k, p, N)
    r0, r1 = rowblock.row_range(m, world, rank)
    ctx = isvd.context(0)
    cb = rowblock.attach_torch(ctx)
    dev = torch.device("cuda", 0)
    s, u, v, it = rowblock.solve_row_block(torch.as_tensor(np.ascontiguousarray(a[r0:r1]), device=dev), k, p, N,
                                           omega=torch.as_tensor(omega, device=dev), integrator=integ,
                                           former=former, tol=tol)
    torch.cuda.synchronize()
    out[rank] = (s.cpu().numpy(), u.cpu().numpy(), v.cpu().numpy(), it, cb.calls, rowblock.allreduces(ctx),
                 repr(cb.error))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("case", CASES, ids=[c[5] for c in CASES])
def test_row_block_ranks_match_single_gpu(cuda, case):
    from mcnla_b200 import isvd
    m, n, k, p, N, integ, former, tol, world = case
    a, omega = _inputs(m, n, k, p, N)
    s1, u1, v1, it1 = isvd.solve(torch.as_tensor(a, device=cuda), k, p, N, omega=torch.as_tensor(omega, device=cuda),
                                 integrator=integ, former=former, tol=tol)
    s1, u1, v1 = s1.cpu().numpy(), u1.cpu().numpy(), v1.cpu().numpy()
    tol_r = TOL
    if integ == "rb_gramian_wy":
        # this integrator moves sigma by ~1e7 times a rounding-level change of A in the reference
        # algorithm itself (its Qbar = Q0 F~ + Qs E~ cancels); the sums over ranks are such a change
        ref = O.isvd(a, omega, k, p, N, integrator=integ, former="svd", tol=tol)
        a1 = a * (1 + 1e-16 * np.random.default_rng(1).standard_normal(a.shape))
        r1 = O.isvd(a1, omega, k, p, N, integrator=integ, former="svd", tol=tol)
        tol_r = max(TOL, 20 * float(np.max(np.abs(r1["s"] - ref["s"]) / ref["s"])))
    tol_vec = TOL if tol_r == TOL else 100 * tol_r     # vectors of the WY case: their own sensitivity
    port = _free_port()
    with mp.get_context("spawn").Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, port, case, out), nprocs=world, join=True)
        res = [out[r] for r in range(world)]
    for r, (s, u, v, it, calls, count, err) in enumerate(res):
        assert err == "None", err
        assert calls > 0 and calls == count, (calls, count)
        assert it == it1, (r, it, it1)
        np.testing.assert_allclose(s, s1, rtol=tol_r)
        assert np.abs(O.align_signs(v, v1) - v1).max() < tol_vec
    u = np.concatenate([x[1] for x in res], axis=0)
    assert u.shape == u1.shape
    assert np.abs(O.align_signs(u, u1) - u1).max() < tol_vec


def test_nccl_communicator_single_rank(cuda):
    """The library's own NCCL communicator on one rank: every reduction point issues an
    ncclAllReduce (counted), and the result is bit for bit the solve without one."""
    from mcnla_b200 import isvd, rowblock
    m, n, k, p, N = 800, 500, 8, 8, 6
    a, omega = _inputs(m, n, k, p, N)
    at, om = torch.as_tensor(a, device=cuda), torch.as_tensor(omega, device=cuda)
    base = isvd.solve(at, k, p, N, omega=om, integrator="rb_gramian_kn", former="rb_gramian", tol=1e-5)
    ctx = isvd.context(cuda)
    rowblock.attach_nccl(ctx, rank=0, world=1)
    try:
        c0 = rowblock.allreduces(ctx)
        got = isvd.solve(at, k, p, N, omega=om, integrator="rb_gramian_kn", former="rb_gramian", tol=1e-5)
        assert rowblock.allreduces(ctx) - c0 == 3      # orthogonalizer W, Bs, former Z
    finally:
        rowblock.detach(ctx)
    assert got[3] == base[3]
    for x, y in zip(got[:3], base[:3]):
        assert torch.equal(x, y)
