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


def test_conv3x3_bounded_wait_runs_out_and_device_stays_usable():
    # A stage barrier that can never complete (it expects 16 bytes more than
    # its loads deliver): the wait gives up after 1 ms, the kernel records
    # code 1 (load wait), lets its copies land, skips its output and returns;
    # the next convolution on the device is correct.
    from feilab_b200 import warmstart
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn((1, 2, 128, 32), generator=g, device="cuda").to(torch.bfloat16)
    w = (torch.randn((9, 32, 32), generator=g, device="cuda") / 17).to(torch.bfloat16)
    assert warmstart.device_error() == 0
    out = warmstart.conv3x3_wait_test(x, w, 1000)
    torch.cuda.synchronize()
    assert warmstart.device_error() == 1
    assert not out.float().abs().any()          # the output was skipped
    again = warmstart.conv3x3(x, w)
    torch.cuda.synchronize()
    assert warmstart.device_error() == 0
    _close(again, _ref_conv(x, None, w, None, False))


def test_conv3x3_rejects_bad_shapes():
    from feilab_b200 import warmstart
    from feilab_b200.icon import IconError
    x = torch.zeros((1, 2, 128, 24), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((9, 16, 24), dtype=torch.bfloat16, device="cuda")
    with pytest.raises(IconError):
        warmstart.conv3x3(x, w)            # 24 channels: not a multiple of 16


# ---------------------------------------------------------------- network
# A plain-PyTorch fp32 mirror of the U-Net (icon_warmstart.h), rounding
# activations to BF16 where the kernels do, so that the library's forward
# pass, its gradients and its training can be checked layer by layer.
LAYERS = [(16, 0, 16), (16, 0, 32), (32, 0, 32), (32, 0, 64), (64, 0, 64), (64, 0, 128), (128, 0, 128),
          (128, 64, 64), (64, 0, 64), (64, 32, 32), (32, 0, 32), (32, 16, 16), (16, 0, 16)]
TOL_NET_REL = 2e-2       # prediction, relative L2 (13 BF16 layers in a row)
TOL_GRAD_COS = 0.99      # per-layer cosine between library and autograd gradients


def _split_params(p):
    out, off = {}, 0
    out["in_w"], out["in_b"] = p[0:144], p[144:160]
    off = 160
    for i, (c0, c1, N) in enumerate(LAYERS):
        n = 9 * N * (c0 + c1)
        out[f"w{i}"], out[f"b{i}"] = p[off:off + n], p[off + n:off + n + N]
        off += n + N
    out["out_w"], out["out_b"] = p[off:off + 16], p[off + 16:off + 17]
    assert off + 17 == p.numel()
    return out


def _mirror(p, Ahwb, gain):
    """Prediction (S, N0, N1) and the network-unit output y (S, Hp, Wp)."""
    import torch.nn.functional as F
    q = _split_params(p)
    bfr = lambda t: t.to(torch.bfloat16).float()
    S, N0, N1 = Ahwb.shape
    Hp, Wp = (N1 + 7) // 8 * 8, (N0 + 7) // 8 * 8
    xr = Ahwb.real.transpose(1, 2)                                  # (S, N1, N0): h = Y, w = X
    sc = torch.sqrt((xr.double() ** 2).mean(dim=(1, 2))).float()
    x = torch.zeros((S, 1, Hp, Wp), device=Ahwb.device)
    x[:, 0, :N1, :N0] = xr / sc[:, None, None]
    w_in = q["in_w"].reshape(3, 3, 16).permute(2, 0, 1)[:, None]   # [16][1][3][3]
    e0a = bfr(torch.relu(F.conv2d(x, w_in, q["in_b"], padding=1)))

    def conv(i, a, b=None):
        c0, c1, N = LAYERS[i]
        w = bfr(q[f"w{i}"]).reshape(3, 3, N, c0 + c1).permute(2, 3, 0, 1)
        inp = a if b is None else torch.cat([a, b], dim=1)
        return bfr(torch.relu(F.conv2d(inp, w, q[f"b{i}"], padding=1)))

    pool = lambda t: bfr(F.avg_pool2d(t, 2))
    up = lambda t: F.interpolate(t, scale_factor=2, mode="nearest")
    e0 = conv(0, e0a)
    e1 = conv(2, conv(1, pool(e0)))
    e2 = conv(4, conv(3, pool(e1)))
    b = conv(6, conv(5, pool(e2)))
    d2 = conv(8, conv(7, up(b), e2))
    d1 = conv(10, conv(9, up(d2), e1))
    d0 = conv(12, conv(11, up(d1), e0))
    y = (d0 * q["out_w"][None, :, None, None]).sum(1) + q["out_b"]
    pred = (sc[:, None, None] * gain * y[:, :N1, :N0]).transpose(1, 2)
    return pred, y, sc, (Hp, Wp)


def _net_case(seed=5, nx=64, thick=40, S=2):
    from feilab_b200 import icon, warmstart
    tilts = np.arange(-48, 49, 4, dtype=np.float32)
    plan = icon.IconPlan(nx, thick, tilts, capacity=4)
    g = torch.Generator(device="cuda").manual_seed(seed)
    re = torch.randn((S, nx, thick), generator=g, device="cuda")
    im = torch.randn((S, nx, thick), generator=g, device="cuda")
    Ahwb = torch.complex(re, im).contiguous()
    net = warmstart.Network(plan, capacity=4)
    net.init(seed)
    return plan, net, Ahwb


import numpy as np  # noqa: E402


def test_network_forward_matches_torch_mirror():
    plan, net, Ahwb = _net_case()
    p, _ = net.get_params()
    net.set_gain(0.5)
    got = net.predict(Ahwb)
    torch.cuda.synchronize()
    from feilab_b200 import warmstart
    assert warmstart.device_error() == 0
    ref, _, _, _ = _mirror(torch.from_numpy(p).cuda(), Ahwb, 0.5)
    rel = ((got - ref).norm() / ref.norm()).item()
    assert rel < TOL_NET_REL, rel


def test_network_gradients_match_autograd():
    plan, net, Ahwb = _net_case(seed=9)
    p, gain = net.get_params()
    g = torch.Generator(device="cuda").manual_seed(11)
    target = torch.randn(Ahwb.shape, generator=g, device="cuda").contiguous()
    loss = net.backprop(Ahwb, target)
    grads = torch.from_numpy(net.grads())
    pt = torch.from_numpy(p).cuda().requires_grad_(True)
    _, y, sc, (Hp, Wp) = _mirror(pt, Ahwb, gain)
    S, N0, N1 = Ahwb.shape
    t = target.transpose(1, 2) / (sc[:, None, None] * gain)
    ref_loss = ((y[:, :N1, :N0] - t) ** 2).mean()
    ref_loss.backward()
    assert abs(loss - ref_loss.item()) <= 2e-2 * ref_loss.item()
    gr = _split_params(pt.grad.detach().cpu())
    gg = _split_params(grads)
    for k in gr:
        a, b = gg[k].double(), gr[k].double()
        cos = (a @ b / (a.norm() * b.norm()).clamp_min(1e-30)).item()
        assert cos > TOL_GRAD_COS, (k, cos)


TOL_GRAD_REL = 1e-1       # per-layer relative L2 of library gradients against the CPU fp32 mirror
TOL_GRAD_ELEM = 2e-1      # every element within this fraction of the layer's largest reference gradient


def test_network_gradients_match_cpu_fp32_mirror():
    """The library's gradients (BF16 activations, FP32 accumulation on the
    tensor cores) against autograd of the fp32 mirror run on the CPU, with
    element-wise bounds per layer."""
    plan, net, Ahwb = _net_case(seed=17)
    p, gain = net.get_params()
    g = torch.Generator(device="cuda").manual_seed(19)
    target = torch.randn(Ahwb.shape, generator=g, device="cuda").contiguous()
    loss = net.backprop(Ahwb, target)
    grads = _split_params(torch.from_numpy(net.grads()))
    A = Ahwb.cpu()
    pt = torch.from_numpy(p).requires_grad_(True)
    _, y, sc, _ = _mirror(pt, A, gain)
    S, N0, N1 = A.shape
    t = target.cpu().transpose(1, 2) / (sc[:, None, None] * gain)
    ref_loss = ((y[:, :N1, :N0] - t) ** 2).mean()
    ref_loss.backward()
    assert abs(loss - ref_loss.item()) <= 2e-2 * ref_loss.item()
    ref = _split_params(pt.grad.detach())
    for k in ref:
        a, b = grads[k].double(), ref[k].double()
        rel = ((a - b).norm() / b.norm().clamp_min(1e-30)).item()
        emax = (a - b).abs().max().item()
        assert rel < TOL_GRAD_REL, (k, rel, emax / max(b.abs().max().item(), 1e-30))
        assert emax <= TOL_GRAD_ELEM * b.abs().max().item() + 1e-12, (k, rel, emax, b.abs().max().item())


def test_network_training_reduces_loss():
    plan, net, Ahwb = _net_case(seed=13)
    # A target the network can represent: a smoothed copy of its input.
    import torch.nn.functional as F
    x = Ahwb.real[:, None]
    target = F.avg_pool2d(x, 3, stride=1, padding=1)[:, 0].contiguous()
    losses = [net.train_step(Ahwb, target, 2e-3) for _ in range(40)]
    torch.cuda.synchronize()
    from feilab_b200 import warmstart
    assert warmstart.device_error() == 0
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])


def test_network_params_round_trip_and_rejects_bad_calls():
    from feilab_b200.icon import IconError
    plan, net, Ahwb = _net_case(seed=17)
    p, _ = net.get_params()
    net.set_params(p * 0.5, gain=2.0)
    q, g = net.get_params()
    assert g == 2.0 and np.array_equal(q, p * 0.5)
    with pytest.raises(IconError):
        net.set_params(p[:-1])
    big = torch.zeros((5,) + tuple(Ahwb.shape[1:]), dtype=torch.complex64, device="cuda")
    with pytest.raises(IconError):
        net.predict(big)                 # beyond the network's capacity of 4
