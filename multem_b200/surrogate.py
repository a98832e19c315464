"""Learned phonon-convergence surrogate: predict the HAADF image averaged over many frozen-phonon
configurations (64) from one averaged over a few (4), with a per-pixel error estimate that gates a
fallback to the plain simulation.

MULTEM has no counterpart: it always averages every configuration explicitly
(Multislice::STEM_ISTEM, src/tem_simulation.cuh:101-200). The network is a stack of 3x3
convolutions (1 -> C -> C -> C -> C -> 2 channels, ReLU between) acting on the scan image divided
by its mean; output channel 0 corrects the input image, channel 1 estimates |error| per pixel.
Forward, backward and the Adam update run in this package's own kernels
(include/multem_b200_surrogate.h: BF16 activations and weights, FP32 accumulation and master
weights); PyTorch only allocates device memory.

    python -m multem_b200.surrogate --train 40 --test 12      # generate, train, evaluate (GPU)

Training data come from the engine itself: for each seeded fcc Au/Pt specimen the 64
configurations are run one at a time, so the 64-configuration image and 16 disjoint
4-configuration images (16 noisy inputs with the same target) come from one simulation.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import api, capi, specimens

WEIGHTS = Path(__file__).resolve().parent / "surrogate_weights.npz"


def _p(t):
    return C.c_void_p(t.data_ptr())


class Net:
    """3x3 conv stack; weights bf16 [Cout, Cin, 3, 3] (+ fp32 master copy), biases fp32."""

    def __init__(self, width=32, depth=5, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = device
        chans = [1] + [width] * (depth - 1) + [2]
        self.layers = list(zip(chans[:-1], chans[1:]))
        g = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for i, (ci, co) in enumerate(self.layers):
            std = (2.0 / (ci * 9)) ** 0.5 * (0.1 if i == len(self.layers) - 1 else 1.0)
            self.w.append((torch.randn(co, ci, 3, 3, generator=g) * std).to(device))
            self.b.append(torch.zeros(co, device=device))
        self.wb = [w.to(torch.bfloat16) for w in self.w]
        self.m = [torch.zeros_like(t) for t in self.w + self.b]
        self.v = [torch.zeros_like(t) for t in self.w + self.b]
        self.step = 0
        self.lib = capi.load()

    # ---- forward / backward through the C ABI ----
    def forward(self, x):
        """x: bf16 [B,1,H,W] -> (activations, head fp32 [B,2,H,W])."""
        torch = self.torch
        B, _, H, W = x.shape
        acts = [x]
        head = None
        for i, (ci, co) in enumerate(self.layers):
            last = i == len(self.layers) - 1
            if last:
                head = torch.empty(B, co, H, W, device=self.dev, dtype=torch.float32)
                capi.check(self.lib.mt_sg_conv3x3_forward(_p(acts[-1]), _p(self.wb[i]), _p(self.b[i]), None, _p(head),
                                                          B, ci, co, H, W, 0, None))
            else:
                y = torch.empty(B, co, H, W, device=self.dev, dtype=torch.bfloat16)
                capi.check(self.lib.mt_sg_conv3x3_forward(_p(acts[-1]), _p(self.wb[i]), _p(self.b[i]), _p(y), None,
                                                          B, ci, co, H, W, 1, None))
                acts.append(y)
        return acts, head

    def train_step(self, x, t, lr=1e-3, lam=0.5):
        torch = self.torch
        B, _, H, W = x.shape
        acts, head = self.forward(x)
        dhead = torch.empty(B, 2, H, W, device=self.dev, dtype=torch.bfloat16)
        terms = torch.empty(B, H, W, device=self.dev, dtype=torch.float32)
        capi.check(self.lib.mt_sg_loss(_p(head), _p(x), _p(t), _p(dhead), _p(terms), B, H, W, float(lam), None))
        grads_w = [None] * len(self.layers)
        grads_b = [None] * len(self.layers)
        dout = dhead
        for i in range(len(self.layers) - 1, -1, -1):
            ci, co = self.layers[i]
            mask = None if i == len(self.layers) - 1 else acts[i + 1]
            dw = torch.empty(co, ci, 3, 3, device=self.dev)
            db = torch.empty(co, device=self.dev)
            capi.check(self.lib.mt_sg_conv3x3_backward_weight(_p(acts[i]), _p(dout), None if mask is None else _p(mask),
                                                              _p(dw), _p(db), B, ci, co, H, W, None))
            grads_w[i], grads_b[i] = dw, db
            if i > 0:
                din = torch.empty(B, ci, H, W, device=self.dev, dtype=torch.bfloat16)
                capi.check(self.lib.mt_sg_conv3x3_backward_data(_p(dout), None if mask is None else _p(mask),
                                                                _p(self.wb[i]), _p(din), B, ci, co, H, W, None))
                dout = din
        self.step += 1
        params = self.w + self.b
        grads = grads_w + grads_b
        for k, (p, g) in enumerate(zip(params, grads)):
            wb = self.wb[k] if k < len(self.w) else None
            capi.check(self.lib.mt_sg_adam(_p(p), None if wb is None else _p(wb), _p(g), _p(self.m[k]), _p(self.v[k]),
                                           p.numel(), float(lr), 0.9, 0.999, 1e-8, self.step, None))
        return float(terms.sum().item()) / terms.numel()

    def predict(self, x):
        """x: bf16 [B,1,H,W] -> (prediction, error estimate), fp32 numpy [B,H,W] each."""
        acts, head = self.forward(x)
        h = head.cpu().numpy()
        xn = x.float().cpu().numpy()[:, 0]
        return xn + h[:, 0], np.abs(h[:, 1])

    def save(self, path=WEIGHTS, **meta):
        d = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        d.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        d["layers"] = np.array(self.layers)
        d["meta"] = np.array(json.dumps(meta))
        np.savez_compressed(path, **d)

    @classmethod
    def load(cls, path=WEIGHTS, device="cuda"):
        import torch
        z = np.load(path)
        layers = [tuple(int(v) for v in r) for r in z["layers"]]
        net = cls(width=layers[0][1], depth=len(layers), device=device)
        for i in range(len(layers)):
            net.w[i] = torch.from_numpy(z[f"w{i}"]).to(device)
            net.b[i] = torch.from_numpy(z[f"b{i}"]).to(device)
        net.wb = [w.to(torch.bfloat16) for w in net.w]
        return net


# ---------------------------------------------------------------------------------------------
# data from the engine

def haadf_specimen(i: int, seed: int = 11, nx: int = 512, ns: int = 32, nconf: int = 64):
    """Seeded fcc(001) Au or Pt specimen (a ~ U[3.92, 4.08] A, thickness ~ U[4, 12] nm, 6 x 6 cells
    wide), 300 kV, 25 mrad probe, one HAADF detector 70-200 mrad, ns x ns raster over 2 x 2 cells,
    `nconf` configurations (sigma 0.085 A), dz_Proj slices of a/2."""
    rng = np.random.default_rng(seed * 100003 + i)
    Z = int(rng.choice((79, 78)))
    a = float(rng.uniform(3.92, 4.08))
    nc = max(2, int(round(rng.uniform(40.0, 120.0) / a)))
    p = specimens.stem_srtio3(nx=nx, ny=nx, na=6, nb=6, nc=nc, ns=ns, nconf=nconf, seed=1 + i)
    p.spec_atoms = specimens.crystal(specimens.fcc_001(Z, a), 6, 6, nc, sigma=0.085)
    p.spec_lx = p.spec_ly = 6 * a
    p.spec_lz = nc * a
    p.spec_dz = a / 2
    p.cond_lens_outer_aper_ang = 25.0
    x0 = 2 * a
    p.scanning_x0, p.scanning_y0 = x0, x0
    p.scanning_xe, p.scanning_ye = x0 + 2 * a, x0 + 2 * a
    p.detector = {"type": 1, "cir": [{"inner_ang": 70.0, "outer_ang": 200.0}]}
    return p


def per_configuration_images(p):
    """HAADF image of each configuration separately ([nconf, ny, nx], each at full weight) and the
    seconds the engine took."""
    e = api.Engine(p)
    n = p.pn_nconf
    out = []
    prev = np.zeros(1)
    t0 = time.perf_counter()
    for c in range(1, n + 1):
        e.run_confs(c, c)
        cur = e.read_stem()[0, 0]
        out.append((cur - prev) * n)
        prev = cur
    dt = time.perf_counter() - t0
    e.close()
    return np.stack(out).transpose(0, 2, 1), dt


def timed_run(p, nconf):
    """Seconds of one plain run of configurations 1..nconf on a set-up engine (set-up excluded)."""
    e = api.Engine(p)
    t0 = time.perf_counter()
    e.run_confs(1, nconf)
    dt = time.perf_counter() - t0
    e.close()
    return dt


def make_pairs(images, n_small=4):
    """Disjoint n_small-configuration means of `images` (nconf x H x W) against their full mean,
    both divided by the small mean's image mean."""
    full = images.mean(axis=0)
    xs, ts = [], []
    for k in range(0, images.shape[0] - n_small + 1, n_small):
        small = images[k:k + n_small].mean(axis=0)
        s = small.mean()
        xs.append(small / s)
        ts.append(full / s)
    return np.stack(xs), np.stack(ts)


def d4(x):
    """The 8 symmetries of the square (fcc(001) images): rotations and mirrors of [.., H, W]."""
    out = []
    for k in range(4):
        r = np.rot90(x, k, axes=(-2, -1))
        out += [r, r[..., ::-1]]
    return out


def rel_rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=40)
    ap.add_argument("--test", type=int, default=12)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--gate", type=float, default=0.02)
    ap.add_argument("--out", default=str(WEIGHTS))
    args = ap.parse_args()
    import torch

    t0 = time.perf_counter()
    train_x, train_t = [], []
    for i in range(args.train):
        imgs, _ = per_configuration_images(haadf_specimen(i))
        x, t = make_pairs(imgs)
        for ax, at in zip(d4(x), d4(t)):
            train_x.append(ax)
            train_t.append(at)
    X = np.ascontiguousarray(np.concatenate(train_x)[:, None], dtype=np.float32)
    T = np.ascontiguousarray(np.concatenate(train_t)[:, None], dtype=np.float32)
    t_gen = time.perf_counter() - t0

    net = Net()
    Xd = torch.from_numpy(X).cuda().to(torch.bfloat16)
    Td = torch.from_numpy(T).cuda()
    rng = np.random.default_rng(0)
    bs = 64
    losses = []
    t1 = time.perf_counter()
    for s in range(args.steps):
        idx = torch.from_numpy(rng.integers(0, X.shape[0], bs)).cuda()
        lr = 2e-3 * (0.5 * (1 + np.cos(np.pi * s / args.steps)))
        losses.append(net.train_step(Xd[idx].contiguous(), Td[idx].contiguous(), lr=lr))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1

    # evaluation on unseen specimens: learned path = 4 configurations + inference (+ fallback)
    res = []
    for i in range(args.train, args.train + args.test):
        p = haadf_specimen(i)
        imgs, _ = per_configuration_images(p)
        n_slices = len(api.specimen_slices(p, 1)["z_0"])
        t_all = timed_run(p, p.pn_nconf)
        t_plain4 = timed_run(haadf_specimen(i, nconf=4), 4)
        small = imgs[:4].mean(axis=0)
        full = imgs.mean(axis=0)
        s = small.mean()
        xd = torch.from_numpy(np.ascontiguousarray((small / s)[None, None], dtype=np.float32)).cuda().to(torch.bfloat16)
        torch.cuda.synchronize()
        ti = time.perf_counter()
        pred, err = net.predict(xd)
        t_inf = time.perf_counter() - ti
        pred, err = pred[0] * s, err[0] * s
        est = float(np.sqrt(np.mean(err ** 2)) / np.sqrt(np.mean(pred ** 2)))
        fallback = est > args.gate
        final = full if fallback else pred
        t_learned = t_plain4 + t_inf + (t_all - t_plain4 if fallback else 0.0)
        n_probes = p.scanning_ns ** 2
        res.append({"n_slices": n_slices, "err_plain4": rel_rms(small, full), "err_learned": rel_rms(pred, full),
                    "err_final": rel_rms(final, full), "est": est, "fallback": bool(fallback),
                    "t_plain64": t_all, "t_learned": t_learned,
                    "updates64": n_probes * p.pn_nconf * n_slices})
    upd = sum(r["updates64"] for r in res)
    summary = {
        "metric": "STEM probe-slice updates/s at 512^2 FP32 (learned: 4 configurations + surrogate, 64-configuration equivalent)",
        "workload": f"{args.test} unseen fcc(001) Au/Pt specimens, 4-12 nm, 512^2 grid, 32x32 HAADF raster (70-200 mrad), "
                    f"300 kV, 25 mrad, 64 phonons",
        "plain_updates_per_s": upd / sum(r["t_plain64"] for r in res),
        "learned_updates_per_s": upd / sum(r["t_learned"] for r in res),
        "rel_rms_error_plain4": float(np.mean([r["err_plain4"] for r in res])),
        "rel_rms_error_learned": float(np.mean([r["err_learned"] for r in res])),
        "rel_rms_error_after_gate": float(np.mean([r["err_final"] for r in res])),
        "max_rel_rms_error_after_gate": float(np.max([r["err_final"] for r in res])),
        "fallback_rate": float(np.mean([r["fallback"] for r in res])),
        "gate": args.gate, "train_specimens": args.train, "train_pairs": int(X.shape[0]),
        "train_steps": args.steps, "final_loss": float(np.mean(losses[-100:])),
        "data_generation_s": round(t_gen, 1), "training_s": round(t_train, 1),
    }
    net.save(args.out, **{k: summary[k] for k in ("workload", "gate", "rel_rms_error_learned")})
    print(json.dumps(summary))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
