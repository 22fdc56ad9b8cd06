"""Learned-preconditioner building blocks on the tcgen05 tensor cores,
checked against plain PyTorch FP32 references of the same ops on the same
BF16-rounded inputs.

3x3 convolution: FP32 accumulation, so channel 0 in FP32 (out32) agrees with
the FP32 reference to 1e-5 relative to the output scale (only the summation
order differs); the BF16 output to BF16 rounding (2^-8 relative)."""
import ctypes as C

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
                                                 (1, 9, 300, 64, 16, 1)])
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
