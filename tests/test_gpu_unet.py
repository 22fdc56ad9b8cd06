"""Learned-preconditioner building blocks on the tcgen05 tensor cores,
checked against plain PyTorch FP32 references of the same ops on the same
BF16-rounded inputs.

3x3 convolution: FP32 accumulation, so channel 0 in FP32 (out32) agrees with
the FP32 reference to 1e-5 relative to the output scale (only the summation
order differs); the BF16 output to BF16 rounding (2^-8 relative)."""
import ctypes as C

import numpy as np

import pytest
import torch
import torch.nn.functional as F

from asd2_b200 import api

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def pack_weights(L, w, cout_pad, cin_pad, stream):
    cout, cin = w.shape[0], w.shape[1]
    wp = torch.empty(L.asd2g_conv_wpack_bytes(cout_pad, cin_pad), dtype=torch.uint8, device="cuda")
    assert L.asd2g_conv_pack_weights(_p(w), cout, cin, cout_pad, cin_pad, _p(wp), C.c_void_p(stream)) == 0
    return wp


@pytest.mark.parametrize("n,h,w,cin,cout,relu", [(1, 8, 128, 16, 16, 0), (2, 20, 200, 16, 32, 1),
                                                 (1, 16, 64, 32, 64, 1), (1, 12, 40, 128, 128, 0),
                                                 (1, 9, 300, 64, 16, 1), (1, 8, 96, 16, 48, 0),
                                                 (1, 8, 136, 32, 96, 1), (1, 6, 64, 48, 192, 0)])
def test_conv3x3_tensor_core(n, h, w, cin, cout, relu):
    L = api.load()
    torch.manual_seed(1)
    s = torch.cuda.current_stream().cuda_stream
    x = torch.randn(n, h, w, cin, device="cuda").to(torch.bfloat16)
    wt = (torch.randn(cout, cin, 3, 3, device="cuda") * 0.2).contiguous()
    b = torch.randn(cout, device="cuda").contiguous()
    wp = pack_weights(L, wt, cout, cin, s)
    out = torch.empty(n, h, w, cout, dtype=torch.bfloat16, device="cuda")
    out32 = torch.empty(n, h, w, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.asd2g_conv3x3_bf16(_p(x), n, h, w, cin, _p(wp), _p(b), cout, _p(out), _p(out32), relu, _p(err),
                              C.c_void_p(s))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = F.conv2d(x.permute(0, 3, 1, 2).float(), wt.to(torch.bfloat16).float(), b, padding=1)
    if relu:
        ref = torch.relu(ref)
    ref = ref.permute(0, 2, 3, 1)
    scale = ref.abs().max().item()
    assert (out32 - ref[..., 0]).abs().max().item() <= 1e-5 * scale
    assert (out.float() - ref).abs().max().item() <= 2 ** -7 * scale


# ------------------------------------------------------------------ U-Net --
def torch_unet(p, x):
    """The same network in PyTorch FP32 (NCHW), from the flat parameter vector."""
    lay, _ = api.UNet.layout()

    def conv(i, t):
        wo, bo, cin, cout, relu = lay[i]
        w = torch.from_numpy(p[wo:wo + cout * cin * 9]).view(cout, cin, 3, 3).cuda()
        b = torch.from_numpy(p[bo:bo + cout]).cuda()
        y = F.conv2d(t, w, b, padding=1)
        return torch.relu(y) if relu else y
    t = x.permute(0, 3, 1, 2)
    e = []
    for lv in range(4):
        ee = conv(2 * lv + 1, conv(2 * lv, t))
        e.append(ee)
        if lv < 3:
            t = F.avg_pool2d(ee, 2)
    low = e[3]
    for lv in (2, 1, 0):
        c = torch.cat([F.interpolate(low, scale_factor=2, mode="nearest"), e[lv]], 1)
        li = 8 + 2 * (2 - lv)
        low = conv(li + 1, conv(li, c))
    return conv(14, low)[:, 0]


def _unet_inputs(B, H, W, seed=0):
    g = torch.Generator(device="cuda").manual_seed(seed)
    feats = torch.rand(B, H, W, 4, device="cuda", generator=g)
    feats[..., 0] = torch.randn(B, H, W, device="cuda", generator=g)
    return feats.contiguous()


def test_unet_forward_matches_fp32_reference():
    B, H, W = 2, 32, 64
    net = api.UNet(B, H, W)
    net.init(seed=3)
    p = net.params()
    feats = _unet_inputs(B, H, W)
    out = torch.empty(B, H, W, device="cuda")
    net.forward(feats, out, B, H, W)
    torch.cuda.synchronize()
    assert net.error_flag() == 0
    ref = torch_unet(p, feats)
    rel = ((out - ref).norm() / ref.norm()).item()
    assert rel < 3e-2, rel  # BF16 activations through 15 layers


def _autograd_unet(pt, feats):
    """The network in PyTorch FP32 with autograd through the flat parameters pt."""
    lay, _ = api.UNet.layout()

    def conv(i, t):
        wo, bo, cin, cout, relu = lay[i]
        y = F.conv2d(t, pt[wo:wo + cout * cin * 9].view(cout, cin, 3, 3), pt[bo:bo + cout], padding=1)
        return torch.relu(y) if relu else y
    t = feats.permute(0, 3, 1, 2)
    e = []
    for lv in range(4):
        ee = conv(2 * lv + 1, conv(2 * lv, t))
        e.append(ee)
        if lv < 3:
            t = F.avg_pool2d(ee, 2)
    low = e[3]
    for lv in (2, 1, 0):
        c = torch.cat([F.interpolate(low, scale_factor=2, mode="nearest"), e[lv]], 1)
        li = 8 + 2 * (2 - lv)
        low = conv(li + 1, conv(li, c))
    return conv(14, low)[:, 0]


def _compare_grads(g, gref, min_cos=0.98):
    lay, _ = api.UNet.layout()
    for i, (wo, bo, cin, cout, relu) in enumerate(lay):
        a, r = g[wo:wo + cout * cin * 9], gref[wo:wo + cout * cin * 9]
        cos = float((a * r).sum() / (np.linalg.norm(a) * np.linalg.norm(r) + 1e-30))
        assert cos > min_cos, (i, cos)
        assert 0.85 < np.linalg.norm(a) / np.linalg.norm(r) < 1.15, (i, np.linalg.norm(a) / np.linalg.norm(r))


def test_unet_gradients_match_autograd():
    B, H, W = 2, 32, 32
    net = api.UNet(B, H, W)
    net.init(seed=5)
    p = net.params()
    feats = _unet_inputs(B, H, W, seed=1)
    target = torch.randn(B, H, W, device="cuda")
    net.train_step(feats, target, B, H, W, lr=0.0)  # gradients of this batch, weights unchanged
    torch.cuda.synchronize()
    g = net.grads()
    assert net.error_flag() == 0
    pt = torch.from_numpy(p).cuda().requires_grad_(True)
    out = _autograd_unet(pt, feats)
    loss = (((out - target) ** 2).sum((1, 2)) / (target ** 2).sum((1, 2))).mean()
    loss.backward()
    _compare_grads(g, pt.grad.cpu().numpy())


def _stencil(feats, v):
    """A v for the symmetric 5-point operator of feats[..., 1:4] (diag,
    coupling to the next row, coupling to the next column)."""
    d, ce, cn = feats[..., 1], feats[..., 2], feats[..., 3]
    y = d * v
    y[:, :-1, :] -= ce[:, :-1, :] * v[:, 1:, :]
    y[:, 1:, :] -= ce[:, :-1, :] * v[:, :-1, :]
    y[:, :, :-1] -= cn[:, :, :-1] * v[:, :, 1:]
    y[:, :, 1:] -= cn[:, :, :-1] * v[:, :, :-1]
    return y


def test_unet_residual_loss_gradients_match_autograd():
    B, H, W = 2, 32, 32
    net = api.UNet(B, H, W)
    net.init(seed=6)
    p = net.params()
    feats = _unet_inputs(B, H, W, seed=4)
    feats[..., 1] += 4.0  # diagonally dominant, like the GFM operator over its scale
    loss_lib = net.train_step_residual(feats, B, H, W, lr=0.0)
    torch.cuda.synchronize()
    g = net.grads()
    assert net.error_flag() == 0
    pt = torch.from_numpy(p).cuda().requires_grad_(True)
    out = _autograd_unet(pt, feats)
    a, r = _stencil(feats, out), feats[..., 0]
    cos2 = (a * r).sum((1, 2)) ** 2 / ((a * a).sum((1, 2)) * (r * r).sum((1, 2)))
    loss = (1.0 - cos2).mean()
    loss.backward()
    assert abs(loss_lib - loss.item()) <= 2e-2 * max(loss.item(), 1e-3) + 1e-3, (loss_lib, loss.item())
    # the output gradient is A (r - c/q a) scaled: a difference of nearly equal
    # terms, rounded to BF16 before the backward pass (0.975 measured at the
    # earliest encoder layer)
    _compare_grads(g, pt.grad.cpu().numpy(), min_cos=0.96)


def test_unet_training_reduces_loss():
    B, H, W = 4, 32, 32
    net = api.UNet(B, H, W)
    net.init(seed=7)
    feats = _unet_inputs(B, H, W, seed=2)
    target = F.avg_pool2d(feats[..., 0].unsqueeze(1), 3, 1, 1).squeeze(1).contiguous()  # a smooth map of the input
    first = net.train_step(feats, target, B, H, W, lr=2e-3)
    last = first
    for _ in range(60):
        last = net.train_step(feats, target, B, H, W, lr=2e-3)
    assert net.error_flag() == 0
    assert last < 0.5 * first, (first, last)


def test_unet_energy_loss_gradients_match_autograd():
    B, H, W = 2, 32, 32
    net = api.UNet(B, H, W)
    net.init(seed=9)
    p = net.params()
    feats = _unet_inputs(B, H, W, seed=5)
    feats[..., 1] += 4.0
    noise = torch.randn(B, 1, H, W, device="cuda", generator=torch.Generator(device="cuda").manual_seed(6))
    target = F.avg_pool2d(F.avg_pool2d(noise, 3, 1, 1), 3, 1, 1)[:, 0].contiguous()  # a smooth error field
    loss_lib = net.train_step_energy(feats, target, B, H, W, lr=0.0)
    torch.cuda.synchronize()
    g = net.grads()
    assert net.error_flag() == 0
    pt = torch.from_numpy(p).cuda().requires_grad_(True)
    out = _autograd_unet(pt, feats)
    ae = _stencil(feats, target)
    pp, q, E = (out * ae).sum((1, 2)), (out * _stencil(feats, out)).sum((1, 2)), (target * ae).sum((1, 2))
    loss = (1.0 - pp ** 2 / (q * E)).mean()
    loss.backward()
    assert abs(loss_lib - loss.item()) <= 2e-2 * max(loss.item(), 1e-3) + 1e-3, (loss_lib, loss.item())
    _compare_grads(g, pt.grad.cpu().numpy(), min_cos=0.96)


def test_unet_residual_training_reduces_loss():
    B, H, W = 4, 32, 32
    net = api.UNet(B, H, W)
    net.init(seed=8)
    feats = _unet_inputs(B, H, W, seed=3)
    feats[..., 1] += 4.0
    first = net.train_step_residual(feats, B, H, W, lr=2e-3)
    last = first
    for _ in range(80):
        last = net.train_step_residual(feats, B, H, W, lr=2e-3)
    assert net.error_flag() == 0
    assert last < 0.6 * first, (first, last)
