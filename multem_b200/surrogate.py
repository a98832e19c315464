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
    """Encoder-decoder of 3x3 convolutions (a U-Net with additive skips).

    With widths (w_0, ..., w_{L-1}) the encoder level l is [pool 2x2 (l > 0)] -> conv(w_l) -> conv(w_l)
    and the decoder level l (l = L-2 ... 0) is upsample 2x -> conv(w_l) -> + encoder output l ->
    conv(w_l); ReLU follows every convolution but the two-channel head conv(2). Images need H and W
    divisible by 2^(L-1). Weights are BF16 [Cout, Cin, 3, 3] with FP32 master copies; biases FP32."""

    def __init__(self, widths=(32, 64, 128, 256), seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.dev = device
        self.widths = tuple(int(w) for w in widths)
        L = len(self.widths)
        convs, cin = [], 1
        for w in self.widths:
            convs += [(cin, w), (w, w)]
            cin = w
        for w in reversed(self.widths[:-1]):
            convs += [(cin, w), (w, w)]
            cin = w
        convs.append((cin, 2))
        self.layers = convs
        self.L = L
        g = torch.Generator().manual_seed(seed)
        self.w, self.b = [], []
        for i, (ci, co) in enumerate(convs):
            std = (2.0 / (ci * 9)) ** 0.5 * (0.1 if i == len(convs) - 1 else 1.0)
            self.w.append((torch.randn(co, ci, 3, 3, generator=g) * std).to(device))
            self.b.append(torch.zeros(co, device=device))
        self.wb = [w.to(torch.bfloat16) for w in self.w]
        self.m = [torch.zeros_like(t) for t in self.w + self.b]
        self.v = [torch.zeros_like(t) for t in self.w + self.b]
        self.step = 0
        self.lib = capi.load()

    def n_params(self):
        return int(sum(t.numel() for t in self.w + self.b))

    # ---- building blocks on the C ABI ----
    def _empty(self, *shape, f32=False):
        t = self.torch
        return t.empty(*shape, device=self.dev, dtype=t.float32 if f32 else t.bfloat16)

    def _conv(self, k, x, relu=True, f32=False):
        B, ci, H, W = x.shape
        co = self.layers[k][1]
        y = self._empty(B, co, H, W, f32=f32)
        capi.check(self.lib.mt_sg_conv3x3_forward(_p(x), _p(self.wb[k]), _p(self.b[k]), None if f32 else _p(y),
                                                  _p(y) if f32 else None, B, ci, co, H, W, int(relu), None))
        return y

    def _resample(self, x, up, scale):
        B, C, H, W = x.shape
        if up:
            y = self._empty(B, C, 2 * H, 2 * W)
            capi.check(self.lib.mt_sg_upsample2(_p(x), _p(y), B, C, H, W, float(scale), None))
        else:
            y = self._empty(B, C, H // 2, W // 2)
            capi.check(self.lib.mt_sg_pool2(_p(x), _p(y), B, C, H, W, float(scale), None))
        return y

    def _add(self, a, b):
        y = self._empty(*a.shape)
        capi.check(self.lib.mt_sg_add(_p(a), _p(b), _p(y), a.numel(), None))
        return y

    def _conv_back(self, k, x, y, g, need_din=True):
        """Gradients of conv k (input x, ReLU output y or None) for the output gradient g."""
        B, ci, H, W = x.shape
        co = self.layers[k][1]
        dw = self._empty(co, ci, 3, 3, f32=True)
        db = self._empty(co, f32=True)
        mask = None if y is None else _p(y)
        capi.check(self.lib.mt_sg_conv3x3_backward_weight(_p(x), _p(g), mask, _p(dw), _p(db), B, ci, co, H, W, None))
        self._gw[k], self._gb[k] = dw, db
        if not need_din:
            return None
        din = self._empty(B, ci, H, W)
        capi.check(self.lib.mt_sg_conv3x3_backward_data(_p(g), mask, _p(self.wb[k]), _p(din), B, ci, co, H, W, None))
        return din

    # ---- forward / backward ----
    def forward(self, x):
        """x: bf16 [B,1,H,W] -> (saved activations, head fp32 [B,2,H,W])."""
        L = self.L
        if x.shape[-1] % (1 << (L - 1)) or x.shape[-2] % (1 << (L - 1)):
            raise ValueError(f"image sides must be multiples of {1 << (L - 1)}")
        enc, saved, h = [], {}, x
        for l in range(L):
            if l > 0:
                h = self._resample(h, False, 0.25)
            a = self._conv(2 * l, h)
            e = self._conv(2 * l + 1, a)
            saved[2 * l], saved[2 * l + 1] = (h, a), (a, e)
            enc.append(e)
            h = e
        k = 2 * L
        for l in range(L - 2, -1, -1):
            u = self._resample(h, True, 1.0)
            d = self._conv(k, u)
            s = self._add(d, enc[l])
            h = self._conv(k + 1, s)
            saved[k], saved[k + 1] = (u, d), (s, h)
            k += 2
        head = self._conv(k, h, relu=False, f32=True)
        saved[k] = (h, None)
        return saved, head

    def backward(self, saved, dhead):
        """Fills the weight and bias gradients for dloss/dhead (bf16 [B,2,H,W])."""
        L = self.L
        n = len(self.layers)
        self._gw, self._gb = [None] * n, [None] * n
        g = self._conv_back(n - 1, *saved[n - 1], dhead)
        skip = {}
        k = n - 3  # decoder level 0 convs are k, k + 1
        for l in range(0, L - 1):
            gs = self._conv_back(k + 1, *saved[k + 1], g)
            skip[l] = gs
            gu = self._conv_back(k, *saved[k], gs)
            g = self._resample(gu, False, 1.0)
            k -= 2
        for l in range(L - 1, -1, -1):
            if l < L - 1:
                g = self._add(g, skip[l])
            ga = self._conv_back(2 * l + 1, *saved[2 * l + 1], g)
            gh = self._conv_back(2 * l, *saved[2 * l], ga, need_din=l > 0)
            if l > 0:
                g = self._resample(gh, True, 0.25)
        return self._gw, self._gb

    def loss_grad(self, head, x, t, lam=0.5):
        B, _, H, W = x.shape
        dhead = self._empty(B, 2, H, W)
        terms = self._empty(B, H, W, f32=True)
        capi.check(self.lib.mt_sg_loss(_p(head), _p(x), _p(t), _p(dhead), _p(terms), B, H, W, float(lam), None))
        return dhead, terms

    def train_step(self, x, t, lr=1e-3, lam=0.5):
        saved, head = self.forward(x)
        dhead, terms = self.loss_grad(head, x, t, lam)
        gw, gb = self.backward(saved, dhead)
        self.step += 1
        for k, (p, g) in enumerate(zip(self.w + self.b, gw + gb)):
            wb = self.wb[k] if k < len(self.w) else None
            capi.check(self.lib.mt_sg_adam(_p(p), None if wb is None else _p(wb), _p(g), _p(self.m[k]), _p(self.v[k]),
                                           p.numel(), float(lr), 0.9, 0.999, 1e-8, self.step, None))
        return float(terms.sum().item()) / terms.numel()

    def predict(self, x):
        """x: bf16 [B,1,H,W] -> (prediction, error estimate), fp32 numpy [B,H,W] each."""
        _, head = self.forward(x)
        h = head.cpu().numpy()
        xn = x.float().cpu().numpy()[:, 0]
        return xn + h[:, 0], np.abs(h[:, 1])

    def save(self, path=WEIGHTS, **meta):
        d = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        d.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        d["widths"] = np.array(self.widths)
        d["meta"] = np.array(json.dumps(meta))
        np.savez_compressed(path, **d)

    @classmethod
    def load(cls, path=WEIGHTS, device="cuda"):
        import torch
        z = np.load(path)
        net = cls(widths=tuple(int(v) for v in z["widths"]), device=device)
        for i in range(len(net.layers)):
            net.w[i] = torch.from_numpy(z[f"w{i}"]).to(device)
            net.b[i] = torch.from_numpy(z[f"b{i}"]).to(device)
        net.wb = [w.to(torch.bfloat16) for w in net.w]
        net.meta = json.loads(str(z["meta"]))
        return net


# ---------------------------------------------------------------------------------------------
# data from the engine

def haadf_specimen(i: int, seed: int = 11, ns: int = 32, scan_cells: int = 2, nconf: int = 64,
                   t_nm=(4.0, 24.0), tilt_deg: float = 2.0):
    """Seeded random fcc(001) Au or Pt specimen: a ~ U[3.92, 4.08] A, thickness ~ U[t_nm] nm, beam
    tilt ~ U[0, tilt_deg] deg at a uniform azimuth; HAADF 70-200 mrad on a 512^2 grid (see
    specimens.haadf_fcc001) with an ns x ns raster over scan_cells x scan_cells unit cells."""
    rng = np.random.default_rng(seed * 100003 + i)
    Z = int(rng.choice((79, 78)))
    a = float(rng.uniform(3.92, 4.08))
    nc = max(2, int(round(rng.uniform(10 * t_nm[0], 10 * t_nm[1]) / a)))
    theta = float(rng.uniform(0.0, tilt_deg))
    phi = float(rng.uniform(0.0, 360.0))
    return specimens.haadf_fcc001(Z, a, nc, nx=512, ns=ns, scan_cells=scan_cells, nconf=nconf, seed=1 + i,
                                  theta=theta, phi=phi)


def per_configuration_images(p):
    """HAADF image of each configuration separately ([nconf, H, W], each at full weight) and the
    seconds each configuration took (set-up of the engine excluded)."""
    e = api.Engine(p)
    n = p.pn_nconf
    out, times = [], []
    prev = np.zeros(1)
    for c in range(1, n + 1):
        t0 = time.perf_counter()
        e.run_confs(c, c)
        cur = e.read_stem()[0, 0]
        times.append(time.perf_counter() - t0)
        out.append((cur - prev) * n)
        prev = cur
    e.close()
    return np.stack(out).transpose(0, 2, 1), np.array(times)


def rel_rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def error_estimate(pred, err):
    """Predicted relative RMS error of an image from the network's per-pixel |error| channel."""
    return float(np.sqrt(np.mean(err ** 2)) / np.sqrt(np.mean(pred ** 2)))


class Surrogate:
    """Trained network plus its gate: predict(small) returns the converged estimate and whether the
    calibrated error estimate stays within the gate (else the caller runs the full simulation)."""

    def __init__(self, net, calib=1.0, gate=0.02):
        self.net, self.calib, self.gate = net, float(calib), float(gate)

    @classmethod
    def load(cls, path=WEIGHTS):
        net = Net.load(path)
        return cls(net, net.meta.get("calib", 1.0), net.meta.get("gate", 0.02))

    def predict(self, small):
        """small: [H, W] HAADF image averaged over a few configurations -> (estimate, predicted
        relative error, accepted)."""
        import torch
        s = float(small.mean())
        x = torch.from_numpy(np.ascontiguousarray((small / s)[None, None], dtype=np.float32)).cuda().to(torch.bfloat16)
        pred, err = self.net.predict(x)
        pred, err = pred[0] * s, err[0] * s
        est = self.calib * error_estimate(pred, err)
        return pred, est, est <= self.gate


def _batches(P, F, rng, bs, n_small):
    """Random training batch: per item a specimen, n_small distinct configurations of it, and one
    of the 8 symmetries of the square applied to the whole batch."""
    import torch
    S, n, H, W = P.shape
    idx = torch.from_numpy(rng.integers(0, S, bs)).cuda()
    sub = torch.from_numpy(np.argsort(rng.random((bs, n)), axis=1)[:, :n_small]).cuda()
    small = P[idx[:, None], sub].mean(dim=1)
    full = F[idx]
    s = small.mean(dim=(1, 2), keepdim=True)
    x, t = small / s, full / s
    k = int(rng.integers(0, 4))
    x, t = torch.rot90(x, k, (1, 2)), torch.rot90(t, k, (1, 2))
    if rng.integers(0, 2):
        x, t = x.flip(2), t.flip(2)
    return x[:, None].contiguous().to(torch.bfloat16), t[:, None].contiguous()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=48, help="training specimens")
    ap.add_argument("--val", type=int, default=4, help="specimens for the gate calibration")
    ap.add_argument("--test", type=int, default=8, help="unseen evaluation specimens")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--gate", type=float, default=0.02)
    ap.add_argument("--test-ns", type=int, default=64, help="evaluation raster (over test-ns/16 unit cells)")
    ap.add_argument("--out", default=str(WEIGHTS))
    args = ap.parse_args()
    import torch

    # training and calibration data: every configuration of each specimen separately
    t0 = time.perf_counter()
    imgs = [per_configuration_images(haadf_specimen(i))[0] for i in range(args.train + args.val)]
    t_gen = time.perf_counter() - t0
    P = torch.from_numpy(np.stack(imgs[:args.train]).astype(np.float32)).cuda()
    F = P.mean(dim=1)

    net = Net()
    rng = np.random.default_rng(0)
    losses = []
    t1 = time.perf_counter()
    for s in range(args.steps):
        x, t = _batches(P, F, rng, args.batch, 4)
        lr = args.lr * 0.5 * (1 + np.cos(np.pi * s / args.steps))
        losses.append(net.train_step(x, t, lr=lr))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1

    # gate calibration on held-out specimens: 16 disjoint 4-configuration inputs each
    raw = Surrogate(net, 1.0, args.gate)
    ratios = []
    for im in imgs[args.train:]:
        full = im.mean(axis=0)
        for k in range(0, im.shape[0], 4):
            pred, est, _ = raw.predict(im[k:k + 4].mean(axis=0))
            ratios.append(rel_rms(pred, full) / est)
    calib = float(np.quantile(ratios, 0.95)) if ratios else 1.0
    sg = Surrogate(net, calib, args.gate)

    # unseen specimens: learned path = 4 configurations + inference (+ the other 60 on fallback)
    res = []
    for i in range(args.train + args.val, args.train + args.val + args.test):
        p = haadf_specimen(i, ns=args.test_ns, scan_cells=max(1, args.test_ns // 16))
        im, tc = per_configuration_images(p)
        n_slices = len(api.specimen_slices(p, 1)["z_0"])
        small, full = im[:4].mean(axis=0), im.mean(axis=0)
        torch.cuda.synchronize()
        ti = time.perf_counter()
        pred, est, ok = sg.predict(small)
        t_inf = time.perf_counter() - ti
        final = pred if ok else full
        t4, t64 = float(tc[:4].sum()), float(tc.sum())
        t_learned = t4 + t_inf + (0.0 if ok else t64 - t4)
        res.append({"n_slices": n_slices, "thickness_A": round(p.spec_lz, 1), "tilt_deg": round(p.theta, 2),
                    "err_plain4": rel_rms(small, full), "err_learned": rel_rms(pred, full),
                    "err_final": rel_rms(final, full), "est": est, "fallback": not ok,
                    "t_plain64_s": t64, "t_plain4_s": t4, "t_inference_s": t_inf, "t_learned_s": t_learned,
                    "updates64": p.scanning_ns ** 2 * p.pn_nconf * n_slices})
    upd = sum(r["updates64"] for r in res)
    summary = {
        "metric": "STEM probe-slice updates/s at 512^2 FP32, learned path (4 configurations + surrogate) "
                  "counted as the 64-configuration run it replaces",
        "workload": f"{args.test} unseen fcc(001) Au/Pt specimens, 4-24 nm, tilt 0-2 deg, 512^2 grid, "
                    f"{args.test_ns}x{args.test_ns} HAADF raster (70-200 mrad), 300 kV, 25 mrad, 64 phonons",
        "plain_updates_per_s": upd / sum(r["t_plain64_s"] for r in res),
        "learned_updates_per_s": upd / sum(r["t_learned_s"] for r in res),
        "rel_rms_error_plain4": float(np.mean([r["err_plain4"] for r in res])),
        "rel_rms_error_learned": float(np.mean([r["err_learned"] for r in res])),
        "rel_rms_error_after_gate": float(np.mean([r["err_final"] for r in res])),
        "max_rel_rms_error_after_gate": float(np.max([r["err_final"] for r in res])),
        "fallback_rate": float(np.mean([r["fallback"] for r in res])),
        "gate": args.gate, "calib": calib, "params": net.n_params(), "widths": list(net.widths),
        "train_specimens": args.train, "train_steps": args.steps, "batch": args.batch,
        "final_loss": float(np.mean(losses[-100:])),
        "data_generation_s": round(t_gen, 1), "training_s": round(t_train, 1),
    }
    net.save(args.out, calib=calib, gate=args.gate, workload=summary["workload"],
             rel_rms_error_learned=summary["rel_rms_error_learned"])
    print(json.dumps(summary))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
