"""Kernels of the learned surrogate (include/multem_b200_surrogate.h) against a PyTorch FP32
reference of the same operations on the same BF16-rounded values, the whole encoder-decoder's
gradients against PyTorch CPU autograd, and a short training run.

Bounds: forward and data gradient 1e-5 relative (FP32 sums of the same products in a different
order), weight gradient 1e-4 (long sums over the batch and image)."""
import ctypes as C

import numpy as np
import pytest

from multem_b200 import capi

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("B,Cin,Cout,H,W", [(2, 3, 5, 20, 37), (3, 8, 16, 32, 32), (1, 16, 2, 16, 16),
                                             (2, 64, 128, 32, 32), (1, 256, 256, 8, 8), (4, 32, 32, 64, 64),
                                             (3, 128, 64, 16, 24)])
def test_conv3x3_forward_and_gradients_match_torch(B, Cin, Cout, H, W):
    torch = pytest.importorskip("torch")
    F = torch.nn.functional
    lib = capi.load()
    g = torch.Generator().manual_seed(B * 100 + Cin)
    x = torch.randn(B, Cin, H, W, generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn(Cout, Cin, 3, 3, generator=g) * 0.3).to(torch.bfloat16).cuda()
    b = torch.randn(Cout, generator=g).cuda()
    # forward with ReLU, bf16 and fp32 outputs
    yb = torch.empty(B, Cout, H, W, device="cuda", dtype=torch.bfloat16)
    yf = torch.empty(B, Cout, H, W, device="cuda")
    capi.check(lib.mt_sg_conv3x3_forward(_p(x), _p(w), _p(b), _p(yb), _p(yf), B, Cin, Cout, H, W, 1, None))
    torch.cuda.synchronize()
    ref = F.relu(F.conv2d(x.float(), w.float(), b, padding=1))
    assert _rel(yf, ref) < 1e-5
    assert _rel(yb.float(), ref) < 1e-2  # BF16 storage
    # gradients through the ReLU: dout masked where the (bf16) output is not positive
    dout = torch.randn(B, Cout, H, W, generator=g).to(torch.bfloat16).cuda()
    xr = x.float().clone().requires_grad_(True)
    wr = w.float().clone().requires_grad_(True)
    br = b.clone().requires_grad_(True)
    out = F.conv2d(xr, wr, br, padding=1)
    mask = (yb.float() > 0).float()
    out.backward(dout.float() * mask)
    din = torch.empty_like(x)
    capi.check(lib.mt_sg_conv3x3_backward_data(_p(dout), _p(yb), _p(w), _p(din), B, Cin, Cout, H, W, None))
    dw = torch.empty(Cout, Cin, 3, 3, device="cuda")
    db = torch.empty(Cout, device="cuda")
    capi.check(lib.mt_sg_conv3x3_backward_weight(_p(x), _p(dout), _p(yb), _p(dw), _p(db), B, Cin, Cout, H, W, None))
    torch.cuda.synchronize()
    assert _rel(din.float(), xr.grad) < 1e-2  # din stored in BF16
    assert _rel(dw, wr.grad) < 1e-4
    assert _rel(db, br.grad) < 1e-4


def test_loss_and_adam_match_their_formulas():
    torch = pytest.importorskip("torch")
    lib = capi.load()
    B, H, W, lam = 2, 16, 16, 0.5
    g = torch.Generator().manual_seed(3)
    head = torch.randn(B, 2, H, W, generator=g).cuda()
    x = torch.rand(B, 1, H, W, generator=g).to(torch.bfloat16).cuda()
    t = torch.rand(B, 1, H, W, generator=g).cuda()
    dh = torch.empty(B, 2, H, W, device="cuda", dtype=torch.bfloat16)
    terms = torch.empty(B, H, W, device="cuda")
    sc = torch.tensor([1.0, 0.5], device="cuda")
    capi.check(lib.mt_sg_loss(_p(head), _p(x), _p(t), _p(sc), _p(dh), _p(terms), B, H, W, lam, None))
    s = sc[:, None, None]
    d = (x.float()[:, 0] + s * head[:, 0] - t[:, 0]) / s
    e = head[:, 1]
    n = B * H * W
    assert _rel(terms, d * d + lam * (e - d.abs()) ** 2) < 1e-6
    assert _rel(dh.float()[:, 0], 2 * d / n) < 1e-2 and _rel(dh.float()[:, 1], 2 * lam * (e - d.abs()) / n) < 1e-2
    w = torch.randn(100, generator=g).cuda()
    w0 = w.clone()
    gr = torch.randn(100, generator=g).cuda()
    m = torch.zeros(100, device="cuda")
    v = torch.zeros(100, device="cuda")
    capi.check(lib.mt_sg_adam(_p(w), None, _p(gr), _p(m), _p(v), 100, 1e-2, 0.9, 0.999, 1e-8, 1, None))
    torch.cuda.synchronize()
    mh, vh = gr, gr * gr  # first step: bias-corrected moments are the gradient and its square
    assert _rel(w, w0 - 1e-2 * mh / (vh.sqrt() + 1e-8)) < 1e-5


class _RoundBF16:
    """Rounds activations to BF16 in the forward pass (the kernels store them in BF16); gradients
    pass unchanged."""

    @staticmethod
    def apply(x):
        import torch
        return x + (x.to(torch.bfloat16).float() - x).detach()


def _torch_reference(net, x, t, lam):
    """The network of multem_b200.surrogate.Net in PyTorch FP32 autograd on the CPU, on the same
    BF16 weights; returns (head, weight gradients, bias gradients)."""
    import torch
    F = torch.nn.functional
    R = _RoundBF16.apply
    W = [w.float().cpu().requires_grad_(True) for w in net.wb]
    Bs = [b.cpu().requires_grad_(True) for b in net.b]
    x, t = x.cpu(), t.cpu()

    def conv(k, h, relu=True):
        y = F.conv2d(h, W[k], Bs[k], padding=1)
        return R(F.relu(y)) if relu else y

    L = net.L
    enc, h = [], x.float()
    for l in range(L):
        if l > 0:
            h = R(F.avg_pool2d(h, 2))
        h = conv(2 * l + 1, conv(2 * l, h))
        enc.append(h)
    k = 2 * L
    for l in range(L - 2, -1, -1):
        u = F.interpolate(h, scale_factor=2, mode="nearest")
        h = conv(k + 1, R(conv(k, u) + enc[l]))
        k += 2
    head = conv(k, h, relu=False)
    d = x.float()[:, 0] + head[:, 0] - t[:, 0]
    loss = (d * d + lam * (head[:, 1] - d.abs().detach()) ** 2).mean()
    loss.backward()
    return head.detach(), [w.grad for w in W], [b.grad for b in Bs]


def test_encoder_decoder_gradients_match_torch_autograd():
    """Forward and every weight/bias gradient of a 3-level encoder-decoder (pooling, upsampling,
    additive skips, ReLU masks) against PyTorch FP32 autograd. Activations and activation
    gradients are BF16 in the kernels, so the bound is 3e-2 relative L2 per tensor; a wrong index,
    mask or missing skip gradient gives errors of order 1."""
    torch = pytest.importorskip("torch")
    from multem_b200.surrogate import Net
    net = Net(widths=(8, 16, 32), in_ch=2, seed=4)
    for b in net.b:  # non-zero biases so that the ReLU masks matter
        b.copy_(torch.randn(b.shape, generator=torch.Generator().manual_seed(b.numel())).cuda() * 0.1)
    g = torch.Generator().manual_seed(5)
    x = (1 + 0.3 * torch.rand(4, 2, 16, 16, generator=g)).to(torch.bfloat16).cuda()
    t = (1 + 0.3 * torch.rand(4, 1, 16, 16, generator=g)).cuda()
    saved, head = net.forward(x)
    dhead, _ = net.loss_grad(head, x, t, lam=0.5)
    gw, gb = net.backward(saved, dhead)
    torch.cuda.synchronize()
    ref_head, rw, rb = _torch_reference(net, x, t, 0.5)
    head, gw, gb = head.cpu(), [v.cpu() for v in gw], [v.cpu() for v in gb]
    assert _rel(head, ref_head) < 1e-2
    for k in range(len(net.layers)):
        assert _rel(gw[k], rw[k]) < 3e-2, f"weight gradient of conv {k}: {_rel(gw[k], rw[k]):.3e}"
        assert _rel(gb[k], rb[k]) < 3e-2, f"bias gradient of conv {k}: {_rel(gb[k], rb[k]):.3e}"


def test_pool_upsample_add_kernels():
    torch = pytest.importorskip("torch")
    F = torch.nn.functional
    lib = capi.load()
    x = torch.randn(2, 3, 8, 12, generator=torch.Generator().manual_seed(1)).to(torch.bfloat16).cuda()
    y = torch.empty(2, 3, 4, 6, device="cuda", dtype=torch.bfloat16)
    capi.check(lib.mt_sg_pool2(_p(x), _p(y), 2, 3, 8, 12, 0.25, None))
    u = torch.empty(2, 3, 16, 24, device="cuda", dtype=torch.bfloat16)
    capi.check(lib.mt_sg_upsample2(_p(x), _p(u), 2, 3, 8, 12, 1.0, None))
    z = torch.empty_like(x)
    capi.check(lib.mt_sg_add(_p(x), _p(x), _p(z), x.numel(), None))
    torch.cuda.synchronize()
    assert _rel(y.float(), F.avg_pool2d(x.float(), 2)) < 4e-3
    assert torch.equal(u.float(), F.interpolate(x.float(), scale_factor=2, mode="nearest"))
    assert torch.equal(z.float(), 2 * x.float())
    assert lib.mt_sg_pool2(_p(x), _p(y), 2, 3, 7, 12, 0.25, None) != 0  # odd height refused


def test_training_reduces_the_loss():
    """A few hundred steps on synthetic data (noisy copies of smooth images) cut the loss."""
    torch = pytest.importorskip("torch")
    from multem_b200.surrogate import Net
    rng = np.random.default_rng(0)
    yy, xx = np.mgrid[0:32, 0:32] / 32.0
    clean = np.stack([1 + 0.5 * np.cos(2 * np.pi * (k % 3 + 1) * xx) * np.cos(2 * np.pi * (k % 2 + 1) * yy)
                      for k in range(64)])
    noisy = clean * (1 + 0.05 * rng.standard_normal(clean.shape))
    X = torch.from_numpy(noisy[:, None].astype(np.float32)).cuda().to(torch.bfloat16)
    T = torch.from_numpy(clean[:, None].astype(np.float32)).cuda()
    net = Net(widths=(16, 32), in_ch=1)
    first = np.mean([net.train_step(X, T, lr=2e-3) for _ in range(5)])
    for _ in range(300):
        last = net.train_step(X, T, lr=2e-3)
    assert last < 0.5 * first


def test_trained_surrogate_gains_over_the_plain_few_configuration_image():
    """What the committed network gains over the method without it, on a specimen outside its
    training, calibration and evaluation sets (fcc Au(001), 16 nm, beam tilted 1.7 deg, 32 x 32
    HAADF raster over 2 x 2 cells, 64 phonon configurations): its estimate from the first 4
    configurations is closer to the 64-configuration image than the plain 4-configuration mean,
    with and without the lattice fold, and so is the folded estimate from 16 configurations; an
    estimate the gate accepts is within twice the gate of the 64-configuration image."""
    pytest.importorskip("torch")
    from multem_b200 import surrogate as S
    sg = S.Surrogate.load()
    im, _ = S.per_configuration_images(S.haadf_specimen(101))
    full = im.mean(axis=0)
    cases = [(4, S.PERIOD), (4, None), (16, S.PERIOD)]
    for n, period in cases:
        small = im[:n].mean(axis=0)
        pred, est, ok = sg.predict(small, n, period)
        e_plain, e_learned = S.rel_rms(small, full), S.rel_rms(pred, full)
        print(f"n={n} fold={bool(period)}: plain {e_plain:.4f} learned {e_learned:.4f} estimate {est:.4f} accepted {ok}")
        assert e_learned < e_plain
        if ok:
            assert e_learned <= 2 * sg.gate
