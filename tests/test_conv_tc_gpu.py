"""The tcgen05 tensor-core convolution of the U-Net (incrmt_conv_bf16,
csrc/conv_tc.cu) against PyTorch's FP32 conv2d of the same BF16 inputs and
weights: every output within 1e-2 of the reference's largest magnitude (the
output is rounded to BF16, a relative step of 2^-8; the FP32 sums differ only
in their order).

The cases cover the three operand swizzles (input channels in chunks of 16,
32 and 64: 32-, 64- and 128-byte rows; 48 and 96 channels run as three
chunks of 16 and of 32), images whose width is not a multiple of the 128-pixel tile (the
partial tiles TMA fills with zeros and the epilogue masks), tiles one row
high (width 128) and eight rows high (width 16), output channels split over
two CTAs (384 = 2 x 192), the 1x1 head, bias and ReLU, and the reversed taps
of the input-gradient convolution; every 3x3 case runs with each kernel
choice (incrmt_conv_set_variant: automatic, one tap per stage, row reuse,
row reuse with the weights resident in persistent CTAs, row reuse with two
128-pixel halves per CTA; the 16 x 8 and 16 x 16 tiles of the last three are
partial at widths 40, 56 and 8 and heights 20 and 12, and the persistent CTAs
each take several tiles of the larger images).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    # batch, H, W, cin, cout, taps, relu, bias, flip
    (2, 32, 48, 16, 32, 9, True, True, False),
    (1, 24, 40, 48, 64, 9, False, True, False),
    (1, 16, 128, 96, 128, 9, True, False, False),
    (2, 16, 16, 128, 16, 9, False, True, False),
    (1, 16, 64, 64, 384, 9, False, False, False),
    (1, 16, 32, 64, 256, 9, True, True, False),
    (2, 32, 32, 32, 16, 1, False, True, False),
    (1, 20, 56, 32, 48, 9, False, False, True),
    (1, 16, 32, 384, 64, 9, False, False, True),
    (1, 12, 8, 32, 32, 9, True, True, False),
    (3, 20, 40, 64, 64, 9, True, True, True),
]


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("B,H,W,cin,cout,taps,relu,use_bias,flip", CASES)
def test_conv_matches_torch(gpu, B, H, W, cin, cout, taps, relu, use_bias, flip, variant):
    import torch
    from incrmt_b200 import capi
    if taps == 1 and variant:
        pytest.skip("the kernel choice concerns 3x3 convolutions")
    capi.conv_set_variant(variant)
    dev = torch.device("cuda")
    g = torch.Generator(device="cpu").manual_seed(B * 1000 + H * 10 + cin + cout + taps)
    x = torch.randn(B, H, W, cin, generator=g).to(torch.bfloat16).to(dev)
    wk = (torch.randn(taps, cout, cin, generator=g) / np.sqrt(taps * cin)).to(torch.bfloat16).to(dev)
    bias = torch.randn(cout, generator=g).to(dev) if use_bias else None
    y = torch.full((B, H, W, cout), float("nan"), dtype=torch.bfloat16, device=dev)
    torch.cuda.synchronize()
    try:
        capi.conv_bf16(x.data_ptr(), B, H, W, cin, wk.data_ptr(), taps, cout, y.data_ptr(),
                       bias.data_ptr() if bias is not None else 0, relu=relu, flip=flip)
        capi.conv_status()
    finally:
        capi.conv_set_variant(0)
    # reference: weights [tap][cout][cin] -> OIHW (tap = 3 ty + tx), taps reversed with flip
    w = wk.float()
    if flip:
        w = torch.flip(w, dims=[0])
    k = 3 if taps == 9 else 1
    wt = w.reshape(k, k, cout, cin).permute(2, 3, 0, 1).contiguous()
    ref = torch.nn.functional.conv2d(x.float().permute(0, 3, 1, 2), wt, bias=bias, padding=k // 2)
    if relu:
        ref = torch.relu(ref)
    ref = ref.permute(0, 2, 3, 1)
    out = y.float()
    assert torch.isfinite(out).all()
    err = (out - ref).abs().max().item() / max(ref.abs().max().item(), 1e-30)
    assert err <= 1e-2, err


WGRAD_CASES = [
    # batch, H, W, cin, cout, taps
    (2, 32, 48, 16, 32, 9),
    (1, 24, 40, 48, 64, 9),
    (1, 16, 128, 96, 128, 9),
    (1, 16, 64, 384, 64, 9),
    (1, 16, 32, 64, 384, 9),
    (2, 32, 32, 32, 16, 1),
]


@pytest.mark.parametrize("B,H,W,cin,cout,taps", WGRAD_CASES)
def test_wgrad_matches_torch(gpu, B, H, W, cin, cout, taps):
    """The weight gradient (incrmt_conv_wgrad_bf16) against torch's
    conv2d_weight in FP32 on the same BF16 values: within 1e-4 of the
    largest entry (the FP32 partial sums differ in order only), added to
    what dW held, and bit for bit the same on a second run."""
    import torch
    from incrmt_b200 import capi
    dev = torch.device("cuda")
    g = torch.Generator(device="cpu").manual_seed(B * 7 + H + W + cin + cout + taps)
    x = torch.randn(B, H, W, cin, generator=g).to(torch.bfloat16).to(dev)
    dy = torch.randn(B, H, W, cout, generator=g).to(torch.bfloat16).to(dev)
    n = capi.conv_wgrad_workspace(B, H, W, cin, cout, taps)
    work = torch.empty(n, dtype=torch.float32, device=dev)
    dw0 = torch.randn(taps, cin, cout, generator=g).to(dev)
    out = []
    for _ in range(2):
        dw = dw0.clone()
        torch.cuda.synchronize()
        capi.conv_wgrad_bf16(x.data_ptr(), dy.data_ptr(), B, H, W, cin, cout, taps, dw.data_ptr(), work.data_ptr(), n)
        capi.conv_status()
        out.append(dw - dw0)
    k = 3 if taps == 9 else 1
    ref = torch.nn.grad.conv2d_weight(x.float().permute(0, 3, 1, 2), (cout, cin, k, k),
                                      dy.float().permute(0, 3, 1, 2), padding=k // 2)
    ref = ref.permute(2, 3, 1, 0).reshape(taps, cin, cout)  # [tap = 3 ty + tx][ci][co]
    err = (out[0] - ref).abs().max().item() / ref.abs().max().item()
    assert err <= 1e-4, err
    assert torch.equal(out[0], out[1])
