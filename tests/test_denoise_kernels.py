"""Numerics of the denoiser's tensor-core kernels against a plain PyTorch
fp32 reference of the same op on the same BF16-rounded inputs.

Tolerance: outputs are BF16 (8-bit mantissa) from FP32 accumulation, so
|gpu - ref| <= 1e-2 * max|ref| + 1e-2 * |ref|; weight gradients stay FP32
(atomics in arbitrary order) and must agree within 2e-3 * max|ref|.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bf(t):
    import torch
    return t.to(torch.bfloat16)


def _pack_w(w, segs, ncols):
    """torch [co][ci][3][3] -> the convolution's BF16 operand [9][K/8][ncols][8]."""
    from relight_b200 import denoise as D
    return D.pack_conv_weights(w, segs, ncols)


def _close(got, ref, rel=1e-2):
    import torch
    got = got.float()
    err = (got - ref).abs()
    lim = rel * ref.abs().max() + rel * ref.abs()
    return bool((err <= lim + 1e-6).all()), float(err.max()), float(ref.abs().max())


@pytest.mark.parametrize("shape", [(2, 20, 37, 16, 9, 32), (1, 64, 64, 64, 64, 128), (3, 9, 8, 32, 32, 16)])
def test_conv3x3_forward(cuda, shape):
    import torch
    from relight_b200 import denoise as D
    n, h, w, cs, cin, co = shape
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.zeros(n, h, w, cs, device="cuda")
    x[..., :cin] = torch.randn(n, h, w, cin, device="cuda", generator=g)
    x = _bf(x)
    wt = _bf(torch.randn(co, cin, 3, 3, device="cuda", generator=g) * 0.2).float()
    b = torch.randn(co, device="cuda", generator=g)
    ncols = (co + 15) // 16 * 16
    wp = _pack_w(wt, [cs], ncols) if cin == cs else _pack_w(torch.nn.functional.pad(wt, (0, 0, 0, 0, 0, cs - cin)), [cs], ncols)
    bias = torch.zeros(ncols, device="cuda")
    bias[:co] = b
    out = torch.zeros(n, h, w, ncols, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D.conv3x3(x, wp, ncols, bias=bias, relu=True, out0=out, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = torch.relu(torch.nn.functional.conv2d(x.float()[..., :cin].permute(0, 3, 1, 2), wt, b, padding=1))
    ok, e, m = _close(out[..., :co].permute(0, 3, 1, 2), ref)
    assert ok, (e, m)


def test_conv3x3_two_segments_split_outputs_masks(cuda):
    """Concatenated inputs (as in the decoder) and two output segments with
    masks (as in the data gradient)."""
    import torch
    from relight_b200 import denoise as D
    n, h, w = 2, 24, 40
    c0, c1, co = 64, 32, 96
    g = torch.Generator(device="cuda").manual_seed(2)
    a = _bf(torch.randn(n, h, w, c0, device="cuda", generator=g))
    bt = _bf(torch.randn(n, h, w, c1, device="cuda", generator=g))
    wt = _bf(torch.randn(co, c0 + c1, 3, 3, device="cuda", generator=g) * 0.1).float()
    wp = _pack_w(wt, [c0, c1], co)
    o0 = torch.zeros(n, h, w, 64, dtype=torch.bfloat16, device="cuda")
    o1 = torch.zeros(n, h, w, 32, dtype=torch.bfloat16, device="cuda")
    m0 = _bf(torch.randn(n, h, w, 64, device="cuda", generator=g))
    m1 = _bf(torch.randn(n, h, w, 32, device="cuda", generator=g))
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D.conv3x3(a, wp, co, in1=bt, out0=o0, out0_c0=0, out0_cn=64, mask0=m0, out1=o1, out1_c0=64,
              out1_cn=32, mask1=m1, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    x = torch.cat([a.float(), bt.float()], -1).permute(0, 3, 1, 2)
    ref = torch.nn.functional.conv2d(x, wt, padding=1).permute(0, 2, 3, 1)
    ref0 = ref[..., :64] * (m0.float() > 0)
    ref1 = ref[..., 64:96] * (m1.float() > 0)
    for got, r in ((o0, ref0), (o1, ref1)):
        ok, e, m = _close(got, r)
        assert ok, (e, m)


@pytest.mark.parametrize("shape", [(2, 20, 37, 32, 16, 9), (4, 16, 16, 128, 128, 96), (1, 33, 17, 16, 128, 128)])
def test_conv3x3_wgrad(cuda, shape):
    import torch
    from relight_b200 import denoise as D
    n, h, w, co, cs, cin = shape
    g = torch.Generator(device="cuda").manual_seed(3)
    gs = (co + 15) // 16 * 16
    grad = torch.zeros(n, h, w, gs, device="cuda")
    grad[..., :co] = torch.randn(n, h, w, co, device="cuda", generator=g)
    grad = _bf(grad)
    x = torch.zeros(n, h, w, cs, device="cuda")
    x[..., :cin] = torch.randn(n, h, w, cin, device="cuda", generator=g)
    x = _bf(x)
    dw = torch.zeros(co, 9, cin + 5, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D.conv3x3_wgrad(grad, co, x, cin, dw, ci_off=5, err=err)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = torch.nn.grad.conv2d_weight(x.float()[..., :cin].permute(0, 3, 1, 2), (co, cin, 3, 3),
                                      grad.float()[..., :co].permute(0, 3, 1, 2), padding=1)
    ref = ref.permute(0, 2, 3, 1).reshape(co, 9, cin)
    e = (dw[..., 5:] - ref).abs().max().item()
    assert e <= 2e-3 * ref.abs().max().item(), (e, ref.abs().max().item())
    assert not dw[..., :5].any()


@pytest.mark.parametrize("c0,c1,co", [(96, 64, 64), (128, 96, 96), (64, 0, 256), (16, 0, 3)])
def test_conv3x3_tile_plans(cuda, c0, c1, co):
    """Each of the convolution's shared-memory plans on odd sizes: weights
    streamed through the ring (96 + 64 -> 64, 128 + 96 -> 96), two issuers of
    256-column accumulators (64 -> 256), and 16 x 16 tiles with a half tile
    past the image's edge (16 -> 3)."""
    import torch
    from relight_b200 import denoise as D
    n, h, w = 1, 21, 27
    g = torch.Generator(device="cuda").manual_seed(4)
    x0 = _bf(torch.randn(n, h, w, c0, device="cuda", generator=g))
    x1 = _bf(torch.randn(n, h, w, c1, device="cuda", generator=g)) if c1 else None
    wt = _bf(torch.randn(co, c0 + c1, 3, 3, device="cuda", generator=g) * 0.05).float()
    b = torch.randn(co, device="cuda", generator=g)
    ncols = (co + 15) // 16 * 16
    wp = _pack_w(wt, [c for c in (c0, c1) if c], ncols)
    bias = torch.zeros(ncols, device="cuda")
    bias[:co] = b
    out = torch.zeros(n, h, w, ncols, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    D.conv3x3(x0, wp, ncols, bias=bias, relu=True, in1=x1, out0=out, err=err, slope=0.1)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    x = torch.cat([x0.float()] + ([x1.float()] if c1 else []), -1).permute(0, 3, 1, 2)
    ref = torch.nn.functional.leaky_relu(torch.nn.functional.conv2d(x, wt, b, padding=1), 0.1)
    ok, e, m = _close(out[..., :co].permute(0, 3, 1, 2), ref)
    assert ok, (e, m)
