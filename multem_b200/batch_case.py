"""Time a batch of uneven simulations (seeded fcc specimens on mixed grids, exit waves and STEM,
frozen phonons; specimens.fcc_batch) through mt_multislice_run_batch against one
mt_multislice_run call per input.

    python -m multem_b200.batch_case --n 32 --workers 4 [--pn-rng 1]

Prints one JSON line: wall times of both, and probe-slice updates/s (STEM: probes x slices x
configurations; exit wave: slices x configurations).
"""
from __future__ import annotations

import argparse
import json
import os
import time


def updates(p, dims_fn):
    import numpy as np
    slices = int(np.ceil(p.spec_lz / p.spec_dz))
    probes = p.scanning_ns ** 2 if p.simulation_type == 11 else 1
    return probes * slices * p.pn_nconf


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--pn-rng", type=int, default=0, help="0 host draws of the reference, 1 device draws")
    args = ap.parse_args()
    os.environ["MTB_BATCH_WORKERS"] = str(args.workers)
    from . import api, specimens

    ps = specimens.fcc_batch(args.n, seed=args.seed)
    for p in ps:
        p.pn_rng = args.pn_rng
    api.ilc_multem(None, ps[1])  # warm-up (STEM) and exit wave
    api.ilc_multem(None, ps[0])
    t0 = time.perf_counter()
    for p in ps:
        api.ilc_multem(None, p)
    t_seq = time.perf_counter() - t0
    t0 = time.perf_counter()
    api.ilc_multem_batch(None, ps)
    t_batch = time.perf_counter() - t0
    n_upd = sum(updates(p, None) for p in ps)
    grids = sorted({p.nx for p in ps})
    print(json.dumps({"workload": f"{args.n} fcc(001) specimens, grids {grids}, EWRS/STEM alternating, "
                                  f"{ps[0].pn_nconf} phonons", "probe_slice_updates": n_upd,
                      "phonon_draws": "device (pn_rng 1)" if args.pn_rng else "host, the reference's (pn_rng 0)",
                      "sequential_s": round(t_seq, 3), "batch_s": round(t_batch, 3),
                      "workers": args.workers, "batch_speedup": round(t_seq / t_batch, 3),
                      "updates_per_s_batch": round(n_upd / t_batch), "updates_per_s_sequential": round(n_upd / t_seq)}))


if __name__ == "__main__":
    main()
