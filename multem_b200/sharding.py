"""Multi-GPU decomposition of a frozen-phonon run: one process per GPU.

Frozen-phonon configurations are independent (Multislice::STEM_ISTEM runs them in sequence and
adds weighted detector sums, src/tem_simulation.cuh:179-198), so each rank takes a contiguous block
of configurations, accumulates its weighted FP64 detector images on its own GPU, and the images are
summed across ranks once at the end (a few hundred KB; no collective inside the loop).
"""
from __future__ import annotations

import numpy as np


def assign_confs(iconf_0: int, iconf_e: int, world: int, rank: int):
    """Contiguous, balanced block [c0, c1] (inclusive, 1-based) of configurations for `rank`;
    (0, -1) when the rank gets none."""
    n = iconf_e - iconf_0 + 1
    base, extra = divmod(n, world)
    start = iconf_0 + rank * base + min(rank, extra)
    count = base + (1 if rank < extra else 0)
    return (start, start + count - 1) if count > 0 else (0, -1)


def reduce_images(img: np.ndarray, dist=None, device=None) -> np.ndarray:
    """Sum FP64 detector images over all ranks (all-reduce); identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return img
    import torch
    t = torch.from_numpy(np.ascontiguousarray(img))
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t)
    return t.cpu().numpy()


def run_stem_sharded(params, dist=None, system_conf=None):
    """Run a STEM simulation with its configurations split over the ranks of `dist`'s default group.
    Returns image_tot [n_thk][n_det][nx][ny] (scan order ix*ny + iy) on every rank."""
    from . import api
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    e = api.Engine(params, system_conf)
    m0 = 1 if not params.pn_single_conf else params.pn_nconf
    c0, c1 = assign_confs(m0, params.pn_nconf if params.pn_model == 3 else 1, world, rank)
    e.reset()
    if c1 >= c0:
        e.run_confs(c0, c1)
    img = e.read_stem()
    e.close()
    dev = None
    if world > 1 and dist.get_backend() == "nccl":
        import torch
        dev = torch.device("cuda", torch.cuda.current_device())
    return reduce_images(img, dist, dev)
