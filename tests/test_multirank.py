"""The multi-GPU mode of this path is replicas only (no exchange step): every
rank runs the same work on its own data and the reported time is the maximum
over ranks.  This test runs that host-side pattern as two gloo ranks on the
CPU: each rank sweeps its own replica of a shell with the oracle, the ranks
all-reduce the maximum of their timings, and every replica must equal the
single-process result bit for bit (no rank depends on another)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _replica(rank, world, port, out_q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import time

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_package
    import oracle

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    msbg = load_package()
    from msbg_rs_b200 import workloads
    sp = workloads.shell_problem(64, 16, seed=1)
    g = msbg.HostGrid("shell", 64, 64, 64, 0.0, 1.0, 16)
    for j, b in enumerate(sp.active):
        g.ensure_block(int(b))
        g.blocks[int(b)][:] = sp.values[j]
    t0 = time.perf_counter()
    oracle.sweep(g, sp.active.astype(np.int64), 0, 0.025, 3, False, threads=1)
    ms = (time.perf_counter() - t0) * 1e3
    t = torch.tensor([ms], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    import hashlib
    digest = hashlib.sha256(np.concatenate([g.blocks[int(b)] for b in sp.active]).tobytes()).hexdigest()
    out_q.put((rank, float(t.item()), ms, digest))
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_agree_and_time_is_max_over_ranks(oracle):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_replica, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][3] == res[1][3]  # identical replicas
    assert res[0][1] == res[1][1] == max(res[0][2], res[1][2])  # every rank sees the max
