"""Multi-process decomposition of a frozen-phonon STEM run (gloo, world size 2, CPU).

Each rank computes its block of configurations with the CPU oracle and the images are all-reduced;
the sum must equal the single-process run (the same decomposition bench.py uses on GPUs with NCCL).
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_q):
    sys.path.insert(0, str(ROOT))
    from multem_b200 import sharding, specimens
    from oracle import runner
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    p = specimens.stem_srtio3(nx=64, ny=64, na=2, nb=2, nc=2, ns=2, nconf=3, seed=5)
    c0, c1 = sharding.assign_confs(1, 3, world, rank)
    img = np.array(runner.stem(p, confs=range(c0, c1 + 1))) if c1 >= c0 else np.zeros((1, 2, 2, 2))
    total = sharding.reduce_images(img, dist)
    if rank == 0:
        out_q.put(total)
    dist.barrier()
    dist.destroy_process_group()


def test_assign_confs_partitions():
    from multem_b200 import sharding
    for n, w in [(16, 1), (16, 2), (16, 3), (5, 8), (1, 2)]:
        seen = []
        for r in range(w):
            c0, c1 = sharding.assign_confs(1, n, w, r)
            seen += list(range(c0, c1 + 1))
        assert seen == list(range(1, n + 1))


def test_two_rank_gloo_reduction_equals_single_run():
    from multem_b200 import specimens
    from oracle import runner
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    total = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    p = specimens.stem_srtio3(nx=64, ny=64, na=2, nb=2, nc=2, ns=2, nconf=3, seed=5)
    ref = np.array(runner.stem(p))
    np.testing.assert_allclose(total, ref, rtol=1e-12, atol=1e-15)
