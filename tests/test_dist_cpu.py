"""The bench's multi-process plumbing on CPU: two gloo ranks on 127.0.0.1 (no GPU).

bench.py under torchrun runs one process per GPU; on more than one rank it only needs a barrier and
the max over ranks of the timed seconds (the solve does not shard: replicas), and the reference arm
runs on rank 0 alone.  Both are exercised here with world_size 2."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _ranks(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier(world)
    m = bench.max_over_ranks(1.5 + rank, world)
    out[rank] = m
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_ranks, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_two_ranks():
    """bench.py --impl reference under torchrun with 2 ranks: rank 0 prints the one JSON line."""
    from oracle import ref_lib
    if not ref_lib.available():
        pytest.skip("oracle/_ref is not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--quick", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
