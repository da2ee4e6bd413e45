"""The learned proposer's tensor-core building blocks against plain PyTorch fp32 references.

A 3x3 convolution layer on tcgen05 (ironav_prop_conv3x3: BF16 operands, FP32 accumulation in TMEM) over
chunk-major padded rasters (each sample a 50 x 50 raster, its 48 x 48 interior and a ring of zeros; channels
in planes of 8) must equal torch's fp32 conv2d of the same BF16 inputs and weights, rounded to BF16: the only
differences are the order of the fp32 sums, so the tolerance is one BF16 rounding step (rtol 1e-2, atol 1e-3).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R = 50


def to_planes(x):
    """[n, C, 48, 48] -> chunk-major padded planes [C/8, n*2500, 8] (contiguous)."""
    import torch

    n, c = x.shape[:2]
    r = torch.zeros((n, R, R, c), dtype=x.dtype, device=x.device)
    r[:, 1:-1, 1:-1, :] = x.permute(0, 2, 3, 1)
    return r.reshape(n * R * R, c // 8, 8).permute(1, 0, 2).contiguous()


def from_planes(p, n):
    c8 = p.shape[0]
    r = p.permute(1, 0, 2).reshape(n, R, R, c8 * 8)
    return r.permute(0, 3, 1, 2)  # [n, C, 50, 50] with the ring


@pytest.mark.parametrize("cin,relu,masked", [(32, 1, False), (16, 1, False), (32, 0, True), (32, 0, False)])
def test_conv3x3_on_tensor_cores_matches_torch(cuda_lib, cin, relu, masked):
    import torch

    lib = cuda_lib
    lib.ironav_prop_conv3x3.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    g = torch.Generator(device="cuda").manual_seed(7 + cin + relu)
    n = 5  # 12500 pixels: 98 tiles of 128, the last one partial
    x = (torch.rand((n, cin, 48, 48), generator=g, device="cuda") * 2 - 1).to(torch.bfloat16)
    w = (torch.randn((9, 32, cin), generator=g, device="cuda") * 0.1).to(torch.bfloat16)
    b = torch.randn(32, generator=g, device="cuda") * 0.1
    xp = to_planes(x)
    yp = torch.full((4, n * R * R, 8), 7.0, dtype=torch.bfloat16, device="cuda")  # every pixel is written
    mask = None
    if masked:
        m = (torch.rand((n, 32, 48, 48), generator=g, device="cuda") > 0.5).to(torch.bfloat16)
        mask = to_planes(m)
    stream = torch.cuda.current_stream().cuda_stream
    st = lib.ironav_prop_conv3x3(xp.data_ptr(), cin, n, w.data_ptr(), b.data_ptr(), relu, mask.data_ptr() if masked else None,
                                 yp.data_ptr(), stream)
    assert st == 0, f"status {st}"
    wt = w.float().reshape(3, 3, 32, cin).permute(2, 3, 0, 1)  # [out, in, dy, dx]
    ref = torch.nn.functional.conv2d(x.float(), wt, b, padding=1)
    if relu:
        ref = torch.relu(ref)
    if masked:
        ref = ref * (from_planes(mask, n)[:, :, 1:-1, 1:-1].float() > 0)
    got = from_planes(yp, n)
    assert torch.all(got[:, :, 0, :] == 0) and torch.all(got[:, :, -1, :] == 0)
    assert torch.all(got[:, :, :, 0] == 0) and torch.all(got[:, :, :, -1] == 0)
    torch.testing.assert_close(got[:, :, 1:-1, 1:-1].float(), ref.to(torch.bfloat16).float(), rtol=1e-2, atol=1e-3)
