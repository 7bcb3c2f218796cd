"""The denoiser network on the tensor cores against a plain PyTorch fp32
copy of the same network (same BF16-rounded parameters and inputs).

Tolerances (the kernels keep activations and gradients in BF16):
  forward output within 5e-2 of the reference's largest magnitude;
  parameter gradients per layer within 8e-2 of that layer's largest
  gradient, and their cosine similarity above 0.99.
A short training run must cut the loss on a learnable toy mapping.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch_net(x, layers):
    """x [n][h][w][16] float -> y [n][h][w][3]; layers = [(w [cout][9][k], b)]."""
    import torch
    import torch.nn.functional as F

    def conv(l, ins, relu=True):
        w, b = layers[l]
        parts = []
        for t in ins:
            c = t.shape[1]
            parts.append(F.pad(t, (0, 0, 0, 0, 0, (c + 63) // 64 * 64 - c)))
        z = torch.cat(parts, 1)
        cout, _, k = w.shape
        wt = w.reshape(cout, 3, 3, k).permute(0, 3, 1, 2)
        o = F.conv2d(z, wt, b, padding=1)
        return F.leaky_relu(o, 0.1) if relu else o

    def pool(t):
        return F.avg_pool2d(t, 2, ceil_mode=True, count_include_pad=False)

    def up(t, like):
        return F.interpolate(t, scale_factor=2, mode="nearest")[:, :, :like.shape[2], :like.shape[3]]

    X = x.permute(0, 3, 1, 2)
    e0 = conv(0, [X])
    e1 = conv(1, [pool(e0)])
    e2 = conv(2, [pool(e1)])
    e3 = conv(3, [pool(e2)])
    d2 = conv(4, [up(e3, e2), e2])
    d1 = conv(5, [up(d2, e1), e1])
    d0 = conv(6, [up(d1, e0), e0])
    y = conv(7, [d0], relu=False)
    return y.permute(0, 2, 3, 1)


def _layers(flat, dev, requires_grad=False):
    import torch
    from relight_b200.denoise import Denoiser
    out = []
    for w, b in Denoiser.unflatten(flat):
        wt = torch.tensor(w, device=dev).to(torch.bfloat16).float().requires_grad_(requires_grad)
        bt = torch.tensor(b, device=dev).requires_grad_(requires_grad)
        out.append((wt, bt))
    return out


def _inputs(n, h, w, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.zeros(n, h, w, 16, device="cuda")
    x[..., :9] = torch.rand(n, h, w, 9, device="cuda", generator=g)
    x[..., 9] = 1.0
    return x.to(torch.bfloat16)


def test_denoiser_forward_matches_torch(cuda):
    import torch
    from relight_b200.denoise import Denoiser
    dn = Denoiser(seed=3)
    x = _inputs(2, 40, 56, 1)
    y = dn.forward(x).float()[..., :3]
    torch.cuda.synchronize()
    assert dn.status() == 0
    ref = _torch_net(x.float(), _layers(dn.params(), "cuda"))
    err = (y - ref).abs().max().item()
    assert err <= 5e-2 * ref.abs().max().item() + 1e-3, (err, ref.abs().max().item())
    dn.close()


def test_denoiser_gradients_match_torch(cuda):
    import torch
    from relight_b200.denoise import Denoiser
    dn = Denoiser(seed=4)
    n, p = 4, 32
    x = _inputs(n, p, p, 2)
    t = torch.zeros(n, p, p, 4, device="cuda")
    t[..., :3] = 5.0   # far from every prediction: the L1 gradient sign is fixed
    t[..., 3] = (torch.rand(n, p, p, device="cuda") < 0.8).float()
    dn.train_step(x, t, lr=-1.0)
    got = dn.grads()
    layers = _layers(dn.params(), "cuda", requires_grad=True)
    y = _torch_net(x.float(), layers)
    pred = y + x.float()[..., :3]
    loss = ((pred - t[..., :3]).abs() * t[..., 3:4]).sum() / (n * p * p * 3)
    loss.backward()
    ref = np.concatenate([np.concatenate([w.grad.cpu().numpy().reshape(-1), b.grad.cpu().numpy()])
                          for w, b in layers])
    o = 0
    for (w, b) in layers:
        k = w.numel() + b.numel()
        g, r = got[o:o + k], ref[o:o + k]
        o += k
        scale = np.abs(r).max()
        assert np.abs(g - r).max() <= 8e-2 * scale + 1e-7, (np.abs(g - r).max(), scale)
        cos = float(g @ r / (np.linalg.norm(g) * np.linalg.norm(r) + 1e-30))
        assert cos > 0.99, cos
    dn.close()


def test_denoiser_training_reduces_loss(cuda):
    """Learn to undo synthetic noise: target = smooth colour, input = it
    plus per-texel noise."""
    import torch
    from relight_b200 import denoise as D
    g = torch.Generator(device="cuda").manual_seed(5)
    n, p = 64, 32
    yy, xx = torch.meshgrid(torch.arange(p, device="cuda"), torch.arange(p, device="cuda"), indexing="ij")
    phase = torch.rand(n, 1, 1, 3, device="cuda", generator=g) * 6.28
    clean = 0.5 + 0.4 * torch.sin(xx[None, :, :, None] * 0.2 + yy[None, :, :, None] * 0.1 + phase)
    noisy = (clean * (1 + 0.8 * torch.randn(n, p, p, 3, device="cuda", generator=g))).clamp_min(0)
    x = torch.zeros(n, p, p, 16, device="cuda")
    x[..., :3] = torch.log1p(noisy)
    x[..., 9] = 1
    t = torch.zeros(n, p, p, 4, device="cuda")
    t[..., :3] = torch.log1p(clean)
    t[..., 3] = 1
    dn = D.Denoiser(seed=6)
    losses = D.train(dn, x.to(torch.bfloat16).contiguous(), t.contiguous(), steps=300, batch=8, lr=3e-3)
    assert dn.status() == 0
    first, last = losses[:20].mean(), losses[-20:].mean()
    assert last < 0.5 * first, (first, last)
    dn.close()
