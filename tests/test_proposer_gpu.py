"""The learned proposer's kernels against plain PyTorch fp32 references of the same operations.

- a 3x3 convolution layer on tcgen05 (ironav_prop_conv3x3: BF16 operands, FP32 accumulation in TMEM) over
  chunk-major padded rasters (each sample a 50 x 50 raster, its 48 x 48 interior and a ring of zeros; channels
  in planes of 8) equals torch's fp32 conv2d of the same BF16 inputs and weights, rounded to BF16: the only
  differences are the order of the fp32 sums, so the tolerance is one BF16 rounding step (rtol 1e-2, atol 1e-3);
- the data gradient (the same kernel with the transposed, mirrored weights and the ReLU mask) equals torch's
  conv2d_input gradient, to the same tolerance;
- the weight and bias gradients on tcgen05 (ironav_prop_wgrad3x3, FP32 outputs) equal torch's conv2d_weight
  gradient and the sum of the output gradient (fp32 sums in another order: rtol 1e-3, atol 1e-3);
- the head's forward and backward passes and the loss's gradient equal torch's autograd of the same
  expressions on the same BF16 features (rtol 1e-4, atol 1e-5, the dz gradient to one BF16 step);
- training steps on a fixed batch reduce its loss.
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
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.ironav_prop_conv3x3(xp.data_ptr(), cin, n, w.data_ptr(), b.data_ptr(), relu, mask.data_ptr() if masked else None,
                                 yp.data_ptr(), err.data_ptr(), stream)
    assert st == 0, f"status {st}"
    assert int(err.item()) == 0
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


@pytest.mark.parametrize("cin", [32, 16])
def test_weight_gradient_on_tensor_cores_matches_torch(cuda_lib, cin):
    import torch

    g = torch.Generator(device="cuda").manual_seed(11 + cin)
    n = 3
    x = (torch.rand((n, cin, 48, 48), generator=g, device="cuda") * 2 - 1).to(torch.bfloat16)
    dz = (torch.rand((n, 32, 48, 48), generator=g, device="cuda") * 2 - 1).to(torch.bfloat16)
    dw = torch.zeros((9, 32, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(32, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xp, zp = to_planes(x), to_planes(dz)  # kept alive: a temporary's memory goes back to the allocator at once
    st = cuda_lib.ironav_prop_wgrad3x3(xp.data_ptr(), cin, zp.data_ptr(), n, dw.data_ptr(), db.data_ptr(), err.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = torch.nn.grad.conv2d_weight(x.float(), (32, cin, 3, 3), dz.float(), padding=1)  # [out, in, dy, dx]
    got = dw.reshape(3, 3, 32, cin).permute(2, 3, 0, 1)
    torch.testing.assert_close(got, ref, rtol=1e-3, atol=1e-3)
    torch.testing.assert_close(db, dz.float().sum(dim=(0, 2, 3)), rtol=1e-3, atol=1e-3)


def test_data_gradient_through_the_relu_matches_torch(cuda_lib):
    """dx = conv2d_input(dz, w) * (x > 0), from ironav_prop_conv3x3 with ironav_prop_weights' transposed weights."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(5)
    n = 4
    w = torch.randn((9, 32, 32), generator=g, device="cuda") * 0.1
    dz = (torch.rand((n, 32, 48, 48), generator=g, device="cuda") * 2 - 1).to(torch.bfloat16)
    xact = torch.relu(torch.rand((n, 32, 48, 48), generator=g, device="cuda") * 2 - 1).to(torch.bfloat16)  # a ReLU output
    wf = torch.zeros((9, 32, 32), dtype=torch.bfloat16, device="cuda")
    wt = torch.zeros_like(wf)
    s = torch.cuda.current_stream().cuda_stream
    assert cuda_lib.ironav_prop_weights(w.data_ptr(), 32, wf.data_ptr(), wt.data_ptr(), s) == 0
    out = torch.zeros((4, n * R * R, 8), dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    zp, ap = to_planes(dz), to_planes(xact)
    assert cuda_lib.ironav_prop_conv3x3(zp.data_ptr(), 32, n, wt.data_ptr(), None, 0, ap.data_ptr(), out.data_ptr(), err.data_ptr(), s) == 0
    torch.cuda.synchronize()
    assert torch.equal(wf.float(), w.to(torch.bfloat16).float())
    wtorch = w.to(torch.bfloat16).float().reshape(3, 3, 32, 32).permute(2, 3, 0, 1)
    ref = torch.nn.grad.conv2d_input((n, 32, 48, 48), wtorch, dz.float(), padding=1) * (xact.float() > 0)
    torch.testing.assert_close(from_planes(out, n)[:, :, 1:-1, 1:-1].float(), ref.to(torch.bfloat16).float(), rtol=1e-2, atol=1e-3)


def test_head_and_loss_match_torch_autograd(cuda_lib):
    import torch

    g = torch.Generator(device="cuda").manual_seed(9)
    n = 6
    feat = torch.relu(torch.randn((n, 32, 48, 48), generator=g, device="cuda")).to(torch.bfloat16)
    hw = torch.randn((13, 32 * 48 * 48), generator=g, device="cuda") * 1e-3
    hb = torch.randn(13, generator=g, device="cuda") * 0.1
    tmv = torch.randint(-128, 128, (n, 2), generator=g, device="cuda").to(torch.int16)
    tpart = torch.randint(0, 5, (n,), generator=g, device="cuda").to(torch.uint8)
    s = torch.cuda.current_stream().cuda_stream
    fp = to_planes(feat)
    out = torch.zeros((n, 13), device="cuda")
    dout = torch.zeros_like(out)
    sums = torch.zeros(3, device="cuda")
    ghw = torch.zeros_like(hw)
    ghb = torch.zeros_like(hb)
    dz = torch.full((4, n * R * R, 8), 3.0, dtype=torch.bfloat16, device="cuda")
    assert cuda_lib.ironav_prop_head_fwd(fp.data_ptr(), n, hw.data_ptr(), hb.data_ptr(), out.data_ptr(), s) == 0
    assert cuda_lib.ironav_prop_loss(out.data_ptr(), tmv.data_ptr(), tpart.data_ptr(), n, dout.data_ptr(), sums.data_ptr(), s) == 0
    assert cuda_lib.ironav_prop_head_bwd(fp.data_ptr(), n, dout.data_ptr(), hw.data_ptr(), ghw.data_ptr(), ghb.data_ptr(), dz.data_ptr(), s) == 0
    torch.cuda.synchronize()
    # the same expressions in torch: features in the head's order (pixel-major, channel-minor)
    f = feat.float().permute(0, 2, 3, 1).reshape(n, -1).requires_grad_(True)
    W = hw.clone().requires_grad_(True)
    B = hb.clone().requires_grad_(True)
    o = f @ W.t() + B
    torch.testing.assert_close(out, o.detach(), rtol=1e-4, atol=1e-5)
    # the packed form of the head (one thread per sample, slices of pixels added atomically): the same sums
    # in another order, so the same FP32 tolerance
    hwt = torch.zeros((32 * 48 * 48, 16), device="cuda")
    out2 = torch.full_like(out, 7.0)
    assert cuda_lib.ironav_prop_head_pack(hw.data_ptr(), hwt.data_ptr(), s) == 0
    assert cuda_lib.ironav_prop_head_fwd_packed(fp.data_ptr(), n, hwt.data_ptr(), hb.data_ptr(), out2.data_ptr(), s) == 0
    torch.cuda.synchronize()
    torch.testing.assert_close(hwt[:, :13], hw.t())
    assert torch.all(hwt[:, 13:] == 0)
    torch.testing.assert_close(out2, o.detach(), rtol=1e-4, atol=1e-5)
    t = tmv.float() / 128.0
    dist = (o[:, :8].reshape(n, 4, 2) - t[:, None, :]).abs().sum(-1)
    lmv = dist.min(dim=1).values + 0.05 * dist.sum(dim=1)
    lce = torch.nn.functional.cross_entropy(o[:, 8:], tpart.long(), reduction="none")
    ((lmv + lce).sum() / n).backward()
    torch.testing.assert_close(sums[0], lmv.sum().detach(), rtol=1e-4, atol=1e-4)
    torch.testing.assert_close(sums[1], lce.sum().detach(), rtol=1e-4, atol=1e-4)
    torch.testing.assert_close(ghw, W.grad, rtol=1e-4, atol=1e-6)
    torch.testing.assert_close(ghb, B.grad, rtol=1e-4, atol=1e-6)
    dfeat = f.grad.reshape(n, 48, 48, 32).permute(0, 3, 1, 2) * (feat.float() > 0)
    got = from_planes(dz, n)
    assert torch.all(got[:, :, 0, :] == 0) and torch.all(got[:, :, :, 0] == 0)
    torch.testing.assert_close(got[:, :, 1:-1, 1:-1].float(), dfeat.to(torch.bfloat16).float(), rtol=1e-2, atol=1e-6)


def test_training_steps_reduce_the_loss_on_a_batch(cuda_lib):
    """The whole step (input, four tcgen05 layers, head, loss, backward through every layer, Adam) on a fixed
    batch of macroblocks of a synthetic sequence with one vector and class for all (targets the network can
    reach from any input): the loss after 40 steps is well below the first."""
    import torch

    from ironav_b200.proposer import SAMPLE_DTYPE, Proposer
    from ironav_b200.synth import Sequence

    seq = Sequence.config("1080p", 2, size=(320, 192))
    f0, f1 = (torch.from_numpy(seq.frame(t)).cuda() for t in range(2))
    mb_w, mb_h = 20, 12
    n = 64
    rng = np.random.default_rng(3)
    idx = rng.choice(mb_w * mb_h, n, replace=False)
    smp = np.zeros(n, dtype=SAMPLE_DTYPE)
    smp["cur"], smp["ref"] = f1.data_ptr(), f0.data_ptr()
    smp["w"], smp["h"], smp["stride"] = 320, 192, 320
    smp["mbx"], smp["mby"] = idx % mb_w, idx // mb_w
    tmv = torch.tensor([[24, -12]] * n, dtype=torch.int16).cuda()
    tpart = torch.ones(n, dtype=torch.uint8).cuda()
    p = Proposer(max_batch=n)
    losses = []
    for _ in range(40):
        p.sums.zero_()
        p.train_step(smp, tmv, tpart, lr=1e-3)
        losses.append(float(p.sums[0] + p.sums[1]) / n)
    p.check_errors()
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.5 * losses[0], losses
