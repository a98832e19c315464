"""Benchmark: STEM probe-slice updates/s at 512^2 FP32.

Workload (the batched STEM ADF case): SrTiO3 (001), a = 3.905 A, 8x8x25 cells (8000 atoms), 300 kV,
21 mrad probe, C3 = 0, defocus 0, 512x512 complex64 grid, dz_Proj slices of 1.95 A (50 slices),
64x64 probe raster over one unit cell (4096 probes, batched 256 per launch), frozen phonons with
per-element sigma (Sr 0.088, Ti 0.075, O 0.095 A), annular detectors 40-80 and 80-200 mrad,
FP32 waves with FP64 detector sums. Synthetic, seeded specimen (no dataset involved).

A step is one frozen-phonon configuration on one GPU: displaced-atom potentials of all 50 slices
(splat + transmission) and all 4096 probes through all 50 slices with detector reduction, i.e.
4096*50 = 204800 probe-slice updates. With N GPUs, one process per GPU (python bench.py --gpus N
starts them itself through torch.distributed.run when it is not already a rank), every rank runs
K configurations of its own block (multem_b200.sharding.assign_confs; weak scaling, no collective
on the data path); the FP64 detector images are all-reduced once at the end and checked against
the sum of the per-rank images. Timing: CUDA events on the engine's stream around the K steps, max
over ranks. The probe batch (512 MiB) exceeds the 126 MB L2, so no flush is needed between steps.

At N = 1, rank 0 also measures, live on the same box, and adds to the line:
  reference_gpu  the reference's own GPU path (Multislice<float, e_device>, cuFFT, per-probe loop,
                 compiled from its sources for sm_100a into oracle/_ref) on samples of this workload;
  learned        the learned phonon-convergence path on an unseen specimen: 4 (then 16)
                 configurations + the surrogate, gated at 2 %, against the 64-configuration run;
  uneven_batch   32 seeded fcc specimens on 256/384/512/1024 grids, exit waves and STEM, 8 phonons,
                 through mt_multislice_run_batch;
  large_field    amorphous carbon on Au(110), 2048^2, 200 kV, 2 A slices: exit-wave slice updates/s.
--no-extras skips them.

--impl reference times the reference's own CPU path (oracle/_ref: MULTEM's Multislice<float, e_host>
compiled from its sources with an FFTW-API shim, as FFTW is not installed) on bounded samples of
the same workload: two raster sizes per step, so that the per-update slope excludes the reference's
per-run set-up; --impl reference --ref-gpu times its GPU path the same way.
--dry-run starts the ranks (gloo on CPU), shards the configurations and runs the final
all-reduce and its check, without any simulation (a check of the multi-process plumbing).
--profile-case NS runs one configuration of the workload with an NS x NS raster (the small case the
ncu captures under profiles/ use: NS = 16 gives one launch of 256 probes, 512 MiB of waves) and
prints its device time; --profile-nx NX runs it on an NX x NX grid instead of 512 x 512.
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
# reference arms (test infrastructure: oracle/_ref is the reference's own code, never ours)

def _raster(p, n_probe_side):
    """An n x n raster with the workload's probe spacing (a / 64), from the same origin."""
    p.scanning_ns = n_probe_side
    p.scanning_xe = p.scanning_ye = p.scanning_x0 + 3.905 * n_probe_side / 64.0
    return p


def cpu_reference_slope(small=2, large=4, nthreads=None):
    """The reference's CPU path on two rasters (small^2 and large^2 probes x 1 phonon x 50 slices of
    the workload). Returns the per-update slope (set-up excluded), the set-up-inclusive rate of the
    larger sample, the seconds spent and a description."""
    from oracle import reference as R
    if not R.available():
        return None
    nthreads = nthreads or os.cpu_count() or 1
    ts = {}
    for n in (small, large):
        p = _raster(workload(1), n)
        t0 = time.perf_counter()
        R.run(p, precision=1, nthreads=nthreads)
        ts[n] = time.perf_counter() - t0
    du = (large * large - small * small) * N_SLICE
    dt = ts[large] - ts[small]
    slope = du / dt if dt > 0 else float("nan")
    incl = large * large * N_SLICE / ts[large]
    desc = (f"reference CPU path (float, {nthreads} threads, FFTW-API shim FFT as FFTW is not installed) on "
            f"{small * small}- and {large * large}-probe rasters x 1 phonon x {N_SLICE} slices of the 512^2 SrTiO3 "
            f"workload; value = per-update slope between the two (the reference's per-run set-up excluded); "
            f"set-up included the larger sample gives {incl:.1f} updates/s")
    return {"slope": slope, "with_setup": incl, "seconds": ts[small] + ts[large], "desc": desc,
            "nthreads": nthreads}


def gpu_reference_slope(small=8, large=32):
    """The reference's own GPU path (Multislice<float, e_device>, cuFFT, per-probe slice loop, built
    for sm_100a into oracle/_ref) on two rasters x 1 phonon x 50 slices of the workload, through its
    run_multislice entry. Returns the per-update slope, the set-up-inclusive rate of the larger
    sample and a description."""
    from oracle import reference as R
    ts = {}
    for n in (small, large):
        p = _raster(workload(1), n)
        t0 = time.perf_counter()
        R.run(p, precision=1, device=True)
        ts[n] = time.perf_counter() - t0
    du = (large * large - small * small) * N_SLICE
    dt = ts[large] - ts[small]
    slope = du / dt if dt > 0 else float("nan")
    incl = large * large * N_SLICE / ts[large]
    desc = (f"reference GPU path (Multislice<float, e_device>: cuFFT, one probe at a time) on the same B200, "
            f"{small * small}- and {large * large}-probe rasters x 1 phonon x {N_SLICE} slices of the 512^2 SrTiO3 "
            f"workload; value = per-update slope (set-up excluded); set-up included the larger sample gives "
            f"{incl:.0f} updates/s")
    return {"slope": slope, "with_setup": incl, "desc": desc}


def _reference_line(args, value, t_all, device, desc, extra):
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_all / max(1, args.steps), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "SrTiO3 (001) 8x8x25, 512^2, 50 slices, 4096-probe raster, 16 phonons "
                                   "(each reference step: two bounded rasters x 1 phonon)",
                       "parallelism": "cpu threads" if device == "cpu" else "1 gpu"},
            "impl": "reference", "device": device, "sample": desc,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    line.update(extra)
    print(json.dumps(line))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import reference as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmultem_ref.so is not built"}))
        return 0
    if args.ref_gpu:
        for _ in range(args.warmup):
            gpu_reference_slope(2, 4)
        rs = [gpu_reference_slope() for _ in range(args.steps)]
        value = statistics.median(r["slope"] for r in rs)
        _reference_line(args, value, 0.0, "gpu", rs[0]["desc"], {})
        return 0
    for _ in range(args.warmup):
        r = R.run(_raster(workload(1), 1), precision=1, nthreads=os.cpu_count() or 1)
    rs = [cpu_reference_slope() for _ in range(args.steps)]
    value = statistics.median(r["slope"] for r in rs)
    t_all = sum(r["seconds"] for r in rs)
    cpu = {"value": value, "unit": UNIT, "cores": rs[0]["nthreads"], "kind": "reference", "sample": rs[0]["desc"]}
    _reference_line(args, value, t_all, "cpu", rs[0]["desc"], {"cpu_baseline": cpu})
    return 0


# ---------------------------------------------------------------------------------------------
# multi-process plumbing

def _free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def relaunch_ranks(args):
    """python bench.py --gpus N outside a torch.distributed launch: start N ranks (one process per
    GPU) through torch.distributed.run on this node, bounded in time."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(Path(__file__).resolve())] + sys.argv[1:]
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", "1")
    try:
        return subprocess.run(cmd, env=env, timeout=args.rank_timeout).returncode
    except subprocess.TimeoutExpired:
        print(json.dumps({"error": f"ranks did not finish within {args.rank_timeout} s"}), file=sys.stderr)
        return 1


def init_ranks(backend):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local, dist


def reduce_and_check(img, dist, device):
    """All-reduce the FP64 detector images once, and check the result against the sum of the
    per-rank images gathered from every rank. Returns (reduced image, max |difference|)."""
    if dist is None:
        return img, 0.0
    import torch
    t = torch.from_numpy(np.ascontiguousarray(img)).to(device)
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    red = t.clone()
    dist.all_reduce(red)
    ref = torch.stack(parts).sum(dim=0)
    diff = float((red - ref).abs().max().item()) if red.numel() else 0.0
    return red.cpu().numpy(), diff


def run_dry(args):
    """Ranks, configuration shards, the final all-reduce and its check, with no simulation."""
    from multem_b200 import sharding
    world, rank, local, dist = init_ranks("gloo")
    per_rank = args.warmup + args.steps
    c0, c1 = sharding.assign_confs(1, per_rank * world, world, rank)
    img = np.zeros((1, 2, 8, 8))
    img[...] = np.arange(c0, c1 + 1).sum()
    red, diff = reduce_and_check(img, dist, "cpu")
    counts = red[0, 0, 0, 0]
    n_all = per_rank * world
    ok = diff == 0.0 and counts == n_all * (n_all + 1) / 2
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": None, "unit": UNIT, "n_gpus": world, "dry_run": True,
                          "steps": args.steps, "warmup": args.warmup, "scaling": "weak",
                          "config": {"parallelism": f"shard{world}", "confs_per_rank": per_rank},
                          "reduce_check": {"max_abs_diff": diff, "ok": bool(ok)}}), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0 if ok else 1


# ---------------------------------------------------------------------------------------------
# our engine

def learned_live(conf):
    """The learned path measured now: an fcc(001) specimen outside the surrogate's training,
    calibration and evaluation sets, 32 x 32 HAADF raster over 2 x 2 cells on a 512^2 grid, its 64
    configurations simulated one by one (engine seconds per configuration). The gated learned path
    runs 4 configurations + the surrogate, then 16, and falls back to all 64 when the calibrated
    error estimate stays above the gate; its result is judged against the 64-configuration image."""
    import torch
    from multem_b200 import api, surrogate
    sg = surrogate.Surrogate.load()
    p = surrogate.haadf_specimen(98, ns=32, scan_cells=2)
    n_slices = len(api.specimen_slices(p, 1)["z_0"])
    im, tc = surrogate.per_configuration_images(p)
    full = im.mean(axis=0)
    out = {"specimen": {"Z": int(p.spec_atoms[0, 0]), "thickness_A": round(float(p.spec_lz), 1),
                        "tilt_deg": round(float(p.theta), 2), "raster": "32x32 over 2x2 cells", "n_slices": n_slices},
           "gate": sg.gate, "noise_floor_of_64_vs_perfect": surrogate.noise_floor(im, 4)}
    upd64 = 32 * 32 * 64 * n_slices
    t64 = float(tc.sum())
    tiers = {}
    used, final, t_inf = 64, full, 0.0
    for n in surrogate.TIERS[:-1]:
        small = im[:n].mean(axis=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pred, est, ok = sg.predict(small, n, surrogate.PERIOD)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        tiers[str(n)] = {"rel_rms_plain": surrogate.rel_rms(small, full), "rel_rms_learned": surrogate.rel_rms(pred, full),
                         "estimate": est, "accepted": bool(ok), "inference_s": dt,
                         "updates_per_s_ungated": upd64 / (float(tc[:n].sum()) + dt)}
        if used == 64:
            t_inf += dt
            if ok:
                used, final = n, pred
    t_learned = float(tc[:used].sum()) + t_inf
    out.update({"tiers": tiers, "configurations_run": used, "rel_rms_result": surrogate.rel_rms(final, full),
                "plain64_updates_per_s": upd64 / t64, "learned_updates_per_s": upd64 / t_learned,
                "speedup_vs_plain64": t64 / t_learned,
                "target": ">= 8x at <= 2 % rel-RMS against the 64-configuration run"})
    return out


def uneven_batch_live(conf):
    """32 seeded fcc(001) specimens on 256/384/512/1024 grids (exit waves and STEM alternating, 8
    phonons each) through one mt_multislice_run_batch call, after one warm-up call of two of them."""
    from multem_b200 import api, specimens
    ps = specimens.fcc_batch(32, seed=3)
    api.ilc_multem_batch(conf, ps[:2])
    t0 = time.perf_counter()
    api.ilc_multem_batch(conf, ps)
    dt = time.perf_counter() - t0
    upd = 0
    for p in ps:
        n_sl = int(math.ceil(p.spec_lz / p.spec_dz))
        upd += (p.scanning_ns ** 2 if p.simulation_type == 11 else 1) * n_sl * p.pn_nconf
    return {"workload": "32 fcc(001) specimens (a 3.8-4.1 A, Z from {13,28,29,46,47,78,79}, 5-30 nm), grids "
                        "256/384/512/1024, 200 or 300 kV, EWRS and STEM (8x8 probes) alternating, 8 phonons",
            "seconds": dt, "probe_slice_updates": upd, "updates_per_s": upd / dt,
            "api": "mt_multislice_run_batch (host in/out, set-up included)"}


def large_field_live(conf):
    """Exit wave of 2 nm amorphous carbon on Au(110) 12x17x60 cells on a 2048^2 grid (200 kV, 2 A
    slices), 8 phonons, through mt_multislice_run after one warm-up call."""
    from multem_b200 import api, specimens
    api.ilc_multem(conf, specimens.au110_amorphous_carbon(nconf=1))
    p = specimens.au110_amorphous_carbon(nconf=8)
    n_sl = len(api.specimen_slices(p, 1)["z_0"])
    t0 = time.perf_counter()
    api.ilc_multem(conf, p)
    dt = time.perf_counter() - t0
    return {"workload": "2 nm a-C on Au(110) 12x17x60 cells (29,292 atoms), 2048^2, 200 kV, 2 A slices, 8 phonons, "
                        "exit wave (EWRS)", "slices": n_sl, "seconds": dt,
            "slice_updates_per_s": 8 * n_sl / dt,
            "api": "mt_multislice_run (host in/out, set-up included)"}


def run_profile_case(args):
    """One configuration of the workload on an NS x NS raster (a bounded case for profilers)."""
    from multem_b200 import api, specimens
    nx = args.profile_nx
    p = _raster(workload(1) if nx == 512 else specimens.stem_srtio3(nx=nx, ny=nx, nconf=1, seed=1), args.profile_case)
    e = api.Engine(p)
    e.prepare_confs(1, 1)
    e.run_prepared(1, 1)
    t = e.timing()
    img = e.read_stem()
    tun = e.tuning()
    n_launch = e.launch_count()
    e.close()
    print(json.dumps({"case": f"{nx}^2 SrTiO3, {args.profile_case}x{args.profile_case} probes, 1 configuration",
                      "device_ms": t["total_ms"], "launches": n_launch, "tuning": tun,
                      "detector_sums": img.sum(axis=(2, 3)).ravel().tolist()}))
    return 0


def run_ours(args):
    world, rank, local, dist = init_ranks("nccl")
    import torch
    from multem_b200 import api, sharding
    from multem_b200.input import SystemConf

    W, K = args.warmup, args.steps
    per_rank = W + K
    n_conf = max(16, per_rank * world)
    p = workload(n_conf)
    conf = SystemConf(precision=1, device=2, gpu_device=local)
    eng = api.Engine(p, conf)
    c0, c1 = sharding.assign_confs(1, per_rank * world, world, rank)
    eng.prepare_confs(c0, c1)                       # host RNG + slicing + uploads (outside timing)
    for c in range(c0, c0 + W):                      # warm-up steps
        eng.run_prepared(c, c)
    eng.reset()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        eng.run_prepared(c0 + W, c1)                 # K timed steps, device-timed inside
        t = eng.timing()
    launches = eng.launch_count()
    variants = eng.pass_variants()
    ms = t["total_ms"]
    img = eng.read_stem()
    reduce_diff = 0.0
    if dist:
        dev = torch.device("cuda", local)
        tt = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
        # the one collective of the run: FP64 detector images summed over the shards
        img, reduce_diff = reduce_and_check(img, dist, dev)
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

    if rank == 0:
        # end to end through the public C ABI: host input struct -> mt_multislice_run -> host output
        ke = max(1, min(K, 2))
        pe = workload(ke, seed=5)
        api.ilc_multem(conf, workload(1, seed=4))  # untimed warm-up call
        calls = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            api.ilc_multem(conf, pe)
            calls.append(time.perf_counter() - t0)
        e2e_val = ke * N_SCAN * N_SLICE / statistics.median(calls)
        n_atoms = 8000
        h2d = n_atoms * 16 + N_SLICE * 8 + (N_SLICE + 1) * (512 + 512) * 8
        d2h = 2 * N_SCAN * 8
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
               "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic",
               "config": {"workload": "SrTiO3 (001) 8x8x25 cells, 8000 atoms, 512^2 grid, 50 slices, "
                                      "64x64 probes (256 per launch), 16+ frozen phonons, 300 kV, 21 mrad, "
                                      "ADF 40-80 & 80-200 mrad", "probes_per_launch": batch,
                          "step": "one phonon configuration (204800 probe-slice updates) per GPU",
                          "l2": "inputs larger than L2 (512 MiB probe batch)", "parallelism": f"shard{world}",
                          "confs_per_rank": K},
               "roofline": {"bound": "hbm", "kernel": f"{dom} line pass", "achieved": achieved, "peak": peak,
                            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                            "algorithmic_bytes_per_launch": bytes_per_launch, "avg_launch_ms": avg,
                            "rows_avg_ms": rows_avg, "cols_avg_ms": cols_avg,
                            "pass_variants": {"rows": "bulk-copy fed" if variants & 1 else "per-thread loads",
                                              "cols": "bulk-copy fed" if variants & 2 else "per-thread loads"}},
               "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "steps": ke, "calls_s": [round(c, 4) for c in calls],
                       "api": "mt_multislice_run (C ABI), host in/out, includes engine set-up; median of 3 calls "
                              "after one warm-up call"},
               "gpu_launches": launches,
               "clocks": clk.summary()}
        if world > 1:
            out["reduce_check"] = {"max_abs_diff": reduce_diff, "image_sum": float(img.sum())}
        if world == 1 and not args.no_extras:
            from oracle import reference as R
            if R.available():
                rg = gpu_reference_slope()
                out["reference_gpu"] = {"value": rg["slope"], "unit": UNIT, "value_with_setup": rg["with_setup"],
                                        "sample": rg["desc"]}
                out["vs_reference_gpu"] = value / rg["slope"]
                out["e2e_vs_reference_gpu"] = e2e_val / rg["slope"]
            for key, fn in (("learned", learned_live), ("uneven_batch", uneven_batch_live),
                            ("large_field", large_field_live)):
                try:
                    out[key] = fn(conf)
                except Exception as exc:  # a leg that cannot run is reported, not hidden
                    out[key] = {"error": f"{type(exc).__name__}: {exc}"}
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_reference_slope()
            if r:
                out["cpu_baseline"] = {"value": r["slope"], "unit": UNIT, "cores": r["nthreads"], "kind": "reference",
                                       "sample": r["desc"], "value_with_setup": r["with_setup"]}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the reference-GPU, learned, uneven-batch and 2048^2 legs")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="with --impl reference: time the reference's own GPU path instead of its CPU path")
    ap.add_argument("--dry-run", action="store_true",
                    help="ranks, shards and the final all-reduce check only (gloo, no GPU work)")
    ap.add_argument("--rank-timeout", type=int, default=1800, help="bound of a self-started multi-rank run (s)")
    ap.add_argument("--profile-case", type=int, default=0, metavar="NS",
                    help="one configuration with an NS x NS raster, for profilers; prints its device time")
    ap.add_argument("--profile-nx", type=int, default=512, metavar="NX",
                    help="grid of the --profile-case run (the same SrTiO3 specimen and slices, NX x NX)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_ranks(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.dry_run:
        return run_dry(args)
    if args.profile_case:
        return run_profile_case(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
