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


def _engine_host_worker(rank, world, port, out_q):
    """Each rank prepares, with the engine's own host model (the C ABI's specimen calls, no GPU), the
    displaced atoms and slicing of the configurations its shard holds."""
    sys.path.insert(0, str(ROOT))
    from multem_b200 import api, sharding, specimens
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    p = specimens.stem_srtio3(nx=64, ny=64, na=2, nb=2, nc=3, ns=2, nconf=5, seed=9)
    c0, c1 = sharding.assign_confs(1, 5, world, rank)
    mine = {}
    for c in range(c0, c1 + 1):
        Z, xyz = api.specimen_atoms(p, c)
        sl = api.specimen_slices(p, c)
        mine[c] = (np.asarray(xyz).copy(), np.asarray(sl["iatom_0"]).copy())
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    if rank == 0:
        out_q.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_engine_host_shards_cover_every_configuration():
    """The shards of two gloo ranks hold every configuration exactly once, and each configuration's
    atoms and slicing prepared on its rank equal those of a single process."""
    from multem_b200 import api, specimens
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_engine_host_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    gathered = q.get(timeout=300)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    seen = [c for part in gathered for c in part]
    assert sorted(seen) == [1, 2, 3, 4, 5]
    p = specimens.stem_srtio3(nx=64, ny=64, na=2, nb=2, nc=3, ns=2, nconf=5, seed=9)
    for part in gathered:
        for c, (xyz, i0) in part.items():
            Z, ref = api.specimen_atoms(p, c)
            np.testing.assert_array_equal(xyz, ref)
            np.testing.assert_array_equal(i0, api.specimen_slices(p, c)["iatom_0"])


def test_bench_starts_two_ranks_by_itself():
    """python bench.py --gpus 2 outside any launcher starts two ranks (torch.distributed.run), which
    shard the configurations and check the final all-reduce; --dry-run runs no simulation, so this
    runs on CPU with gloo."""
    import json
    import subprocess
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", "--dry-run", "--steps", "2"],
                       capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["dry_run"] and d["reduce_check"]["ok"]
