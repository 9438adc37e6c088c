"""The iSVD drivers of the reference (src/isvd_dense_rb.cpp, src/isvd_dense_cb.cpp) on the B200.

    python -m mcnla_b200.isvd_dense <A-file> <S-file> <U-file> <V-file>
        [#sketch] [rank] [over-sampling-rank] [tolerance] [maxiter]
        [--layout rb|cb] [--integrator NAME] [--former NAME] [--seed S] [--binary]

The positional arguments and their defaults are the reference drivers' (N = 16, k = 20,
p = 12, tol = 1e-3, maxiter = 256; src/isvd_dense_rb.cpp:66-94).  A is read from a dense
MatrixMarket file into pinned host memory and solved through the host-buffer entry point
(mcnla_b200_isvd_host), which copies a large row-major A to the device in row blocks behind the
sketch.  An MCNLA dense binary file (--binary, row-block layout) is streamed instead: its row
blocks are read into the library's pinned staging buffers while the device copies and sketches
the previous ones (mcnla_b200_isvd_stream).  The stages default to the drivers'
choices: the row-block driver's Gramian orthogonalizer, row-block Wen-Yin integrator and
row-block Gramian former (src/isvd_dense_rb.cpp:12-34); --layout cb keeps A column-major and
uses the column-block Gramian former (src/isvd_dense_cb.cpp:20-34).  Omega is drawn from the
Gaussian generator the drivers seed with rand(); here --seed (default: the clock) seeds the
device generator, and Omega is copied to the device with A.

S, U and V are written as the drivers write them (saveMatrixMarket, src/isvd_dense_rb.cpp:
254-274), and the drivers' check ||A - U S V'||_F / ||A||_F (src/isvd_dense_rb.cpp:291-315) is
printed with the stage times and the iteration count.

Under torchrun with several ranks (one GPU each) the matrix is split by rows as the reference
splits it over MPI ranks: every rank reads its row block, the stages sum their partial products
through the library's NCCL communicator, and rank 0 gathers U and writes the files.
"""
import argparse
import os
import sys
import time

import numpy as np

INTEGRATORS = ["kn", "rb_kn", "rb_gramian_kn", "rb_wy", "rb_gramian_wy"]
FORMERS = ["svd", "gramian", "rb_gramian", "cb_gramian"]


def parse(argv=None):
    ap = argparse.ArgumentParser(prog="python -m mcnla_b200.isvd_dense",
                                 description="iSVD of a dense matrix file (the reference's isvd_dense drivers)")
    ap.add_argument("a_file")
    ap.add_argument("s_file")
    ap.add_argument("u_file")
    ap.add_argument("v_file")
    ap.add_argument("num_sketch", nargs="?", type=float, default=16)
    ap.add_argument("rank", nargs="?", type=float, default=20)
    ap.add_argument("over_rank", nargs="?", type=float, default=12)
    ap.add_argument("tolerance", nargs="?", type=float, default=1e-3)
    ap.add_argument("maxiter", nargs="?", type=float, default=256)
    ap.add_argument("--layout", choices=["rb", "cb"], default="rb")
    ap.add_argument("--integrator", choices=INTEGRATORS, default="rb_wy")
    ap.add_argument("--former", choices=FORMERS, default=None)
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--binary", action="store_true", help="A is an MCNLA dense binary file")
    args = ap.parse_args(argv)
    args.num_sketch, args.rank, args.over_rank, args.maxiter = (int(args.num_sketch), int(args.rank),
                                                               int(args.over_rank), int(args.maxiter))
    if args.former is None:
        args.former = "cb_gramian" if args.layout == "cb" else "rb_gramian"
    if args.seed is None:
        args.seed = int(time.time())
    return args


def load_a(args, rows=None):
    """A (or rows = (first, count) of it) in pinned host memory: row-major for the row-block
    driver, column-major (its transpose buffer) for the column-block one."""
    import torch
    from . import io
    if args.binary:
        dims, vt = io.binary_size(args.a_file)
        if len(dims) != 2:
            raise ValueError("A must be a matrix")
        # the reference's row-major matrix has dims {n, m} (contiguous along a row)
        cm = args.layout == "cb"
        m, n = (dims[0], dims[1]) if cm else (dims[1], dims[0])
        if rows is not None and cm:
            raise ValueError("row blocks of a column-major binary file are not contiguous")
        first, count = rows if rows is not None else (0, dims[-1])
        host = io.load_binary(args.a_file, first, count).reshape(count, dims[0])
        a = host if not cm else host          # cm: the n x m buffer is A column-major
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory(), m, n
    m, n, _ = io.matrix_market_size(args.a_file)
    if args.layout == "cb":
        a = io.load_matrix_market(args.a_file, order="F")
        buf = np.ascontiguousarray(a.T)       # n x m: A column-major
        return torch.from_numpy(buf).pin_memory(), m, n
    a = io.load_matrix_market(args.a_file, rows=rows)
    return torch.from_numpy(a).pin_memory(), m, n


def frobenius_error(a_dev, s, u, v, colmajor=False):
    """||A - U S V'||_F^2 and ||A||_F^2 of this rank's rows (the drivers' check), on the device."""
    import torch
    a = a_dev.t() if colmajor else a_dev
    num = den = 0.0
    for r0 in range(0, a.shape[0], 8192):
        blk = a[r0:r0 + 8192]
        num += float(((blk - (u[r0:r0 + 8192] * s) @ v.t()) ** 2).sum().item())
        den += float((blk * blk).sum().item())
    return num, den


def frobenius_error_stream(read_rows, m, n, s, u, v, block=8192):
    """The drivers' check for a streamed A: the file's row blocks read again into pinned memory
    and compared on the device block by block."""
    import torch
    buf = torch.empty(min(block, m), n, dtype=torch.float64, pin_memory=True)
    num = den = 0.0
    for r0 in range(0, m, block):
        rows = min(block, m - r0)
        read_rows(r0, rows, buf.data_ptr())
        blk = buf[:rows].to(u.device)
        num += float(((blk - (u[r0:r0 + rows] * s) @ v.t()) ** 2).sum().item())
        den += float((blk * blk).sum().item())
    return num, den


def main(argv=None):
    args = parse(argv)
    import torch
    from . import io, isvd, rowblock, synthetic
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    k, p, N = args.rank, args.over_rank, args.num_sketch
    l = k + p
    if world > 1:
        import datetime
        import torch.distributed as dist
        if args.layout == "cb":
            raise SystemExit("the row-block decomposition over ranks reads row blocks: use --layout rb")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        m, n, _ = io.matrix_market_size(args.a_file) if not args.binary else (None, None, None)
        if args.binary:
            dims, _ = io.binary_size(args.a_file)
            m, n = dims[1], dims[0]
        r0, r1 = rowblock.row_range(m, world, rank)
        a_host, _, _ = load_a(args, rows=(r0, r1 - r0))
    elif args.binary and args.layout == "rb":
        # streamed ingest: the file's row blocks go to the device behind the sketch
        m, n, read_rows = io.binary_row_reader(args.a_file)
        a_host = None
        r0, r1 = 0, m
    else:
        a_host, m, n = load_a(args)
        r0, r1 = 0, m
    if rank == 0:
        print("MCNLA-compatible iSVD driver for DenseMatrix on the B200 (%s version)"
              % ("row-block" if args.layout == "rb" else "column-block"))
        print("m = %d, n = %d, k = %d, p = %d, N = %d, tol = %g, maxiter = %d" % (m, n, k, p, N, args.tolerance,
                                                                              args.maxiter))
        print("%d GPU(s) / %s; stages: GaussianProjection / Gramian / %s / %s"
              % (world, torch.cuda.get_device_name(dev), args.integrator, args.former))
    omega = synthetic.omega_torch(n, l * N, seed=args.seed, device=dev)
    omega_host = omega.cpu().pin_memory()
    t0 = time.perf_counter()
    if world > 1:
        ctx = isvd.context(dev)
        rowblock.attach_nccl(ctx, rank=rank, world=world)
        a_dev = a_host.to(dev, non_blocking=True)
        s, u, v, it = isvd.solve(a_dev, k, p, N, omega=omega, integrator=args.integrator, former=args.former,
                                 maxit=args.maxiter, tol=args.tolerance)
        torch.cuda.synchronize()
    elif a_host is None:
        s, u, v, it = isvd.solve_stream(read_rows, m, n, omega_host, k, p, N, integrator=args.integrator,
                                        former=args.former, maxit=args.maxiter, tol=args.tolerance, device=dev)
        s, u, v = s.to(dev), u.to(dev), v.to(dev)
    else:
        s, u, v, it = isvd.solve_host(a_host, omega_host, k, p, N, integrator=args.integrator, former=args.former,
                                      maxit=args.maxiter, tol=args.tolerance, colmajor=args.layout == "cb",
                                      device=dev)
        a_dev = a_host.to(dev)
        s, u, v = s.to(dev), u.to(dev), v.to(dev)
    elapsed = time.perf_counter() - t0
    if a_host is None:
        num, den = frobenius_error_stream(read_rows, m, n, s, u, v)
    else:
        num, den = frobenius_error(a_dev, s, u, v, colmajor=args.layout == "cb")
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([num, den], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        num, den = float(t[0]), float(t[1])
        blocks = [torch.empty(rowblock.row_range(m, world, r)[1] - rowblock.row_range(m, world, r)[0], k,
                              dtype=torch.float64, device=dev) for r in range(world)]
        dist.all_gather(blocks, u.contiguous())
        u = torch.cat(blocks)
    if rank == 0:
        print("Total computing time:  %.6f seconds (files excluded)" % elapsed)
        print("Iteration = %d" % it)
        print("Error     = %.6e" % (num / den) ** 0.5)
        print("Error := norm(A - Uk Sk Vk')_F / norm(A)_F")
        print("Write S into %s." % args.s_file)
        io.save_matrix_market(args.s_file, s.cpu().numpy().reshape(-1, 1))
        print("Write U into %s." % args.u_file)
        io.save_matrix_market(args.u_file, u.cpu().numpy())
        print("Write V into %s." % args.v_file)
        io.save_matrix_market(args.v_file, v.cpu().numpy())
    if world > 1:
        import torch.distributed as dist
        rowblock.detach(isvd.context(dev))
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
