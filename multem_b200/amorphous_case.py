"""Run the amorphous-carbon-on-Au(110) exit-wave workload (specimens.au110_amorphous_carbon: 2048^2
grid, 12 x 17 x 60 Au(110) cells under 2 nm of a-C, 200 kV, 2 A slices, frozen phonons) once
through mt_multislice_run and print one JSON line with the slice count and the wall time.

    python -m multem_b200.amorphous_case --nconf 32
"""
from __future__ import annotations

import argparse
import json
import time


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nconf", type=int, default=32)
    ap.add_argument("--nx", type=int, default=2048)
    args = ap.parse_args()
    import numpy as np

    from . import api, specimens

    p = specimens.au110_amorphous_carbon(nx=args.nx, ny=args.nx, nconf=args.nconf)
    n_slices = len(api.specimen_slices(p, 1)["z_0"])
    api.ilc_multem(None, specimens.au110_amorphous_carbon(nx=args.nx, ny=args.nx, nconf=1))  # warm-up
    t0 = time.perf_counter()
    out = api.ilc_multem(None, p)
    dt = time.perf_counter() - t0
    psi = out["data"][0]["psi_coh"]
    print(json.dumps({"workload": f"Au(110) 12x17x60 + 2 nm a-C, {args.nx}^2, 200 kV, {args.nconf} phonons",
                      "atoms": int(len(p.spec_atoms)), "slices": n_slices, "seconds": round(dt, 3),
                      "slice_updates_per_s": round(args.nconf * n_slices / dt, 1),
                      "mean_intensity": float(np.mean(np.abs(psi) ** 2))}))


if __name__ == "__main__":
    main()
