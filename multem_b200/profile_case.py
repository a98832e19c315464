"""Run a bounded slice of the 512^2 SrTiO3 STEM workload once through the C ABI (for profilers).

    python -m multem_b200.profile_case --ns 16 --batch 128

runs one phonon configuration with an ns x ns probe raster in batches of `batch` probes
(batch * 2 MiB of probe waves on the device) and prints the device time.
"""
from __future__ import annotations

import argparse
import os


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ns", type=int, default=16)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--nx", type=int, default=512)
    args = ap.parse_args()
    os.environ["MTB_BATCH"] = str(args.batch)
    from . import api, specimens

    p = specimens.stem_srtio3(nx=args.nx, ny=args.nx, nconf=1)
    a = 3.905
    p.scanning_ns = args.ns
    p.scanning_xe = p.scanning_x0 + a * args.ns / 64.0
    p.scanning_ye = p.scanning_y0 + a * args.ns / 64.0
    e = api.Engine(p)
    e.prepare_confs(1, 1)
    e.run_prepared(1, 1)
    t = e.timing()
    img = e.read_stem()
    print(f"probes {args.ns * args.ns}, batch {args.batch}: {t['total_ms']:.2f} ms, launches {e.launch_count()}, "
          f"detector sums {img.sum(axis=(2, 3)).ravel().tolist()}")
    e.close()


if __name__ == "__main__":
    main()
