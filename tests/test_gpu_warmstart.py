"""Tensor-core convolution and warm-start network against plain PyTorch fp32.

The kernels compute in BF16 with FP32 accumulation and round outputs to
BF16, so they are compared with torch's fp32 convolution of the same BF16
inputs at a BF16 tolerance: relative L2 error below 4e-3 and every element
within 2^-7 of the reference's largest magnitude (output rounding is 2^-9
relative).
"""
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL_REL_L2 = 4e-3
TOL_ABS_FRAC = 2.0 ** -7


def _ref_conv(in0, in1, w, bias, relu):
    import torch.nn.functional as F
    x = in0.float() if in1 is None else torch.cat([in0.float(), in1.float()], dim=3)
    N = w.shape[1]
    wt = w.float().reshape(3, 3, N, -1).permute(2, 3, 0, 1)    # [N][C][dy][dx], tap = 3*dy + dx
    y = F.conv2d(x.permute(0, 3, 1, 2), wt, bias, padding=1).permute(0, 2, 3, 1)
    return torch.relu(y) if relu else y


def _close(got, ref):
    got = got.float()
    rel = ((got - ref).norm() / ref.norm().clamp_min(1e-30)).item()
    mx = (got - ref).abs().max().item()
    assert rel < TOL_REL_L2, rel
    assert mx <= TOL_ABS_FRAC * ref.abs().max().item() + 1e-6, mx


CASES = [
    # n, H, W, c0, c1, N, relu, bias
    (2, 5, 130, 16, 0, 16, True, True),      # ragged width, 32-byte swizzle
    (1, 3, 256, 32, 0, 32, False, True),     # 64-byte swizzle
    (1, 4, 128, 64, 0, 128, True, True),     # 128-byte swizzle, N = 128
    (1, 3, 128, 128, 64, 64, True, True),    # concatenated input (decoder level 3)
    (1, 3, 200, 32, 16, 16, True, False),    # concatenated, 16-channel chunks
    (1, 2, 128, 64, 0, 192, False, False),   # N = 192
    (1, 2, 64, 128, 0, 256, False, False),   # N = 256, width below one tile
]


@pytest.mark.parametrize("n,H,W,c0,c1,N,relu,use_bias", CASES)
def test_conv3x3_matches_torch(n, H, W, c0, c1, N, relu, use_bias):
    from feilab_b200 import warmstart
    g = torch.Generator(device="cuda").manual_seed(1000 + c0 + N)
    dev = "cuda"
    in0 = torch.randn((n, H, W, c0), generator=g, device=dev).to(torch.bfloat16)
    in1 = torch.randn((n, H, W, c1), generator=g, device=dev).to(torch.bfloat16) if c1 else None
    w = (torch.randn((9, N, c0 + c1), generator=g, device=dev) / (3 * (c0 + c1) ** 0.5)).to(torch.bfloat16)
    bias = torch.randn((N,), generator=g, device=dev) * 0.1 if use_bias else None
    out = warmstart.conv3x3(in0, w, bias, relu, in1=in1)
    torch.cuda.synchronize()
    assert warmstart.device_error() == 0
    _close(out, _ref_conv(in0, in1, w, bias, relu))


def test_conv3x3_split_and_accumulate():
    # Output channels split over two tensors, the second accumulated (the
    # gradient of a concatenated input added to a skip branch's gradient).
    from feilab_b200 import warmstart
    g = torch.Generator(device="cuda").manual_seed(7)
    n, H, W, C, N, ns = 2, 3, 160, 32, 48, 32
    x = torch.randn((n, H, W, C), generator=g, device="cuda").to(torch.bfloat16)
    w = (torch.randn((9, N, C), generator=g, device="cuda") / 17).to(torch.bfloat16)
    prev = torch.randn((n, H, W, N - ns), generator=g, device="cuda").to(torch.bfloat16)
    out1 = prev.clone()
    out0, out1 = warmstart.conv3x3(x, w, None, False, nsplit=ns, out1=out1, acc1=True)
    torch.cuda.synchronize()
    assert warmstart.device_error() == 0
    ref = _ref_conv(x, None, w, None, False)
    _close(out0, ref[..., :ns])
    _close(out1, ref[..., ns:] + prev.float())


def test_conv3x3_repeatable():
    from feilab_b200 import warmstart
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn((1, 4, 256, 64), generator=g, device="cuda").to(torch.bfloat16)
    w = (torch.randn((9, 64, 64), generator=g, device="cuda") / 24).to(torch.bfloat16)
    a = warmstart.conv3x3(x, w)
    b = warmstart.conv3x3(x, w)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_conv3x3_rejects_bad_shapes():
    from feilab_b200 import warmstart
    from feilab_b200.icon import IconError
    x = torch.zeros((1, 2, 128, 24), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((9, 16, 24), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(IconError):
        warmstart.conv3x3(x, w)            # 24 channels: not a multiple of 16
