"""Benchmark: STEM probe-slice updates/s at 512^2 FP32.

Workload (the batched STEM ADF case): SrTiO3 (001), a = 3.905 A, 8x8x25 cells (8000 atoms), 300 kV,
21 mrad probe, C3 = 0, defocus 0, 512x512 complex64 grid, dz_Proj slices of 1.95 A (50 slices),
64x64 probe raster over one unit cell (4096 probes, batched 256 per launch), frozen phonons with
per-element sigma (Sr 0.088, Ti 0.075, O 0.095 A), annular detectors 40-80 and 80-200 mrad,
FP32 waves with FP64 detector sums. Synthetic, seeded specimen (no dataset involved).

A step is one frozen-phonon configuration on one GPU: displaced-atom potentials of all 50 slices
(splat + transmission) and all 4096 probes through all 50 slices with detector reduction, i.e.
4096*50 = 204800 probe-slice updates. With N GPUs (torchrun), every rank runs K configurations of
its own (weak scaling; shards are independent, no collective on the data path); the detector
images are reduced once at the end. Timing: CUDA events on the engine's stream around the K steps,
max over ranks. The probe batch (512 MiB) exceeds the 126 MB L2, so no flush is needed between
steps.

--impl reference times the reference's own CPU path (oracle/_ref: MULTEM's Multislice<float, e_host>
compiled from its sources with an FFTW-API shim) on a bounded sample of the same workload;
--impl reference --ref-gpu times the reference's own GPU path (Multislice<float, e_device>, built for
sm_100a into the same library) on 1024-probe samples instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "STEM probe-slice updates/s at 512^2 FP32 (plain)"
UNIT = "probe-slice updates/s"
N_SLICE = 50
N_SCAN = 4096
NXY = 512 * 512
BYTES_PER_UPDATE = 32 * NXY  # psi read + written once in each of the two passes


def measured_peak_gbs():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "ncu_line_passes_512.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def workload(n_conf, seed=1):
    from multem_b200 import specimens
    return specimens.stem_srtio3(nconf=n_conf, seed=seed)


# ---------------------------------------------------------------------------------------------
def cpu_reference_sample(n_probe_side=2, nthreads=None):
    """Reference CPU path on a bounded sample of the workload: same specimen, grid and slices, one
    phonon configuration, a n x n probe raster. Returns (updates/s, seconds, sample description)."""
    from oracle import reference as R
    if not R.available():
        return None
    nthreads = nthreads or os.cpu_count() or 1
    p = workload(1)
    p.scanning_ns = n_probe_side
    a = 3.905
    x0 = p.scanning_x0
    p.scanning_xe = p.scanning_ye = x0 + a * n_probe_side / 64.0
    t0 = time.perf_counter()
    R.run(p, precision=1, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n_upd = n_probe_side * n_probe_side * N_SLICE
    desc = (f"{n_probe_side * n_probe_side} probes x 1 phonon x {N_SLICE} slices of the 512^2 SrTiO3 workload "
            f"(includes the reference's per-run set-up)")
    return n_upd / dt, dt, desc, nthreads


def gpu_reference_sample(n_probe_side):
    """The reference's own GPU path (Multislice<float, e_device>, cuFFT, built for sm_100a into
    oracle/_ref) on an n x n probe raster x 1 phonon x 50 slices of the workload, through its
    run_multislice entry (set-up included, as a caller of ilc_multem pays it)."""
    from oracle import reference as R
    p = workload(1)
    p.scanning_ns = n_probe_side
    a = 3.905
    p.scanning_xe = p.scanning_ye = p.scanning_x0 + a * n_probe_side / 64.0
    t0 = time.perf_counter()
    R.run(p, precision=1, device=True)
    return time.perf_counter() - t0


def run_reference_gpu(args):
    ns = 32
    for _ in range(args.warmup):
        gpu_reference_sample(4)
    t_all = sum(gpu_reference_sample(ns) for _ in range(args.steps))
    value = args.steps * ns * ns * N_SLICE / t_all
    sample = (f"{ns * ns} probes x 1 phonon x {N_SLICE} slices of the 512^2 SrTiO3 workload per step, through the "
              f"reference's GPU path (float, cuFFT, per-probe slice loop), set-up included")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_all / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "SrTiO3 (001) 8x8x25, 512^2, 50 slices, 4096-probe raster, 16 phonons "
                                   f"(each reference step: {ns * ns} probes x 1 phonon)", "parallelism": "1 gpu"},
            "impl": "reference", "device": "gpu", "sample": sample,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import reference as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmultem_ref.so is not built"}))
        return 0
    if args.ref_gpu:
        return run_reference_gpu(args)
    for _ in range(args.warmup):
        cpu_reference_sample(1)
    vals = []
    t_all = 0.0
    for _ in range(args.steps):
        v, dt, desc, nth = cpu_reference_sample(2)
        vals.append(v)
        t_all += dt
    value = len(vals) * 4 * N_SLICE / t_all
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_all / len(vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "SrTiO3 (001) 8x8x25, 512^2, 50 slices, 4096-probe raster, 16 phonons "
                                   "(each reference step: 4 probes x 1 phonon)", "parallelism": "cpu threads"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "reference", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------------
def run_ours(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from multem_b200 import api
    from multem_b200.input import SystemConf

    W, K = args.warmup, args.steps
    per_rank = W + K
    n_conf = max(16, per_rank * world)
    p = workload(n_conf)
    conf = SystemConf(precision=1, device=2, gpu_device=local)
    eng = api.Engine(p, conf)
    c0 = rank * per_rank + 1
    eng.prepare_confs(c0, c0 + per_rank - 1)       # host RNG + slicing + uploads (outside timing)
    for c in range(c0, c0 + W):                      # warm-up steps
        eng.run_prepared(c, c)
    eng.reset()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        eng.run_prepared(c0 + W, c0 + per_rank - 1)  # K timed steps, device-timed inside
        t = eng.timing()
    launches = eng.launch_count()
    variants = eng.pass_variants()
    ms = t["total_ms"]
    if dist:
        tt = torch.tensor([ms], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        # final FP64 reduction of the detector images across shards (one collective per run)
        img = torch.from_numpy(eng.read_stem()).to(f"cuda:{local}")
        dist.all_reduce(img)
        dist.barrier()
    total_updates = world * K * N_SCAN * N_SLICE
    value = total_updates / (ms / 1e3)

    # roofline of the dominant line pass (separate timed step with per-launch events)
    eng.set_timing(True)
    eng.run_prepared(c0 + W, c0 + W)
    kt = eng.timing()
    eng.set_timing(False)
    batch = int(os.environ.get("MTB_BATCH", "256"))
    bytes_per_launch = 16 * NXY * batch       # one pass over a batch: read + write complex64
    rows_avg = kt["rows_ms"] / max(1, kt["n_rows"])
    cols_avg = kt["cols_ms"] / max(1, kt["n_cols"])
    dom = "rows" if kt["rows_ms"] >= kt["cols_ms"] else "cols"
    avg = rows_avg if dom == "rows" else cols_avg
    peak, peak_kind = measured_peak_gbs()
    achieved = bytes_per_launch / (avg / 1e3) / 1e9
    prof = profile_traffic()
    traffic = None
    if prof and dom in prof:
        traffic = prof[dom].get("dram_bytes_per_launch_scaled")

    eng.close()  # its device memory returns to the library's pool, which the next engine reuses

    out = None
    if rank == 0:
        # end to end through the public C ABI: host input struct -> mt_multislice_run -> host output
        ke = max(1, min(K, 2))
        pe = workload(ke, seed=5)
        api.ilc_multem(conf, workload(1, seed=4))  # untimed warm-up call
        calls = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = api.ilc_multem(conf, pe)
            calls.append(time.perf_counter() - t0)
        e2e_val = ke * N_SCAN * N_SLICE / statistics.median(calls)
        n_atoms = 8000
        h2d = n_atoms * 16 + N_SLICE * 8 + (N_SLICE + 1) * (512 + 512) * 8
        d2h = 2 * N_SCAN * 8 // 1
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_reference_sample(2)
            if r:
                v, dt, desc, nth = r
                cpu = {"value": v, "unit": UNIT, "cores": nth, "kind": "reference", "sample": desc}
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
               "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic",
               "config": {"workload": "SrTiO3 (001) 8x8x25 cells, 8000 atoms, 512^2 grid, 50 slices, "
                                      "64x64 probes (256 per launch), 16+ frozen phonons, 300 kV, 21 mrad, "
                                      "ADF 40-80 & 80-200 mrad", "probes_per_launch": batch,
                          "step": "one phonon configuration (204800 probe-slice updates) per GPU",
                          "l2": "inputs larger than L2 (512 MiB probe batch)", "parallelism": f"shard{world}"},
               "roofline": {"bound": "hbm", "kernel": f"{dom} line pass", "achieved": achieved, "peak": peak,
                            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                            "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg,
                            "rows_avg_ms": rows_avg, "cols_avg_ms": cols_avg,
                            "pass_variants": {"rows": "bulk-copy fed" if variants & 1 else "per-thread loads",
                                              "cols": "bulk-copy fed" if variants & 2 else "per-thread loads"}},
               "cpu_baseline": cpu,
               "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "steps": ke, "calls_s": [round(c, 4) for c in calls],
                       "api": "mt_multislice_run (C ABI), host in/out, includes engine set-up; median of 3 calls "
                              "after one warm-up call"},
               "gpu_launches": launches,
               "clocks": clk.summary(),
               "learned": learned_record()}
        print(json.dumps(out), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def learned_record():
    """The learned path's figures as measured when the committed surrogate was evaluated (HAADF,
    fcc(001) Au/Pt, 512^2 grid, 10 unseen specimens, 64 configurations as the reference result);
    they are not re-timed in this run."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "multem_b200", "surrogate_weights.npz")
    if not os.path.exists(path):
        return None
    import numpy as np
    meta = json.loads(str(np.load(path)["meta"]))
    keys = ("plain_updates_per_s", "learned_updates_per_s", "learned4_updates_per_s", "rel_rms_error_learned4",
            "rel_rms_error_learned16", "rel_rms_error_plain4", "max_rel_rms_error_after_gate", "fallback_rate",
            "rel_rms_error_floor4")
    return {"source": "recorded by python -m multem_b200.surrogate (profiles/surrogate_haadf_fcc001_512.md); "
                      "not timed in this run",
            "workload": meta.get("workload"), "gate": meta.get("gate"),
            "crystal_mode": {k: meta.get(f"crystal_{k}") for k in keys},
            "generic_mode": {k: meta.get(f"generic_{k}") for k in keys}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="with --impl reference: time the reference's own GPU path instead of its CPU path")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
