"""Tensor-core convolution layers of the warm-start network against torch's
FP32 convolutions on the same bf16 values (forward, data and weight
gradients), and one network forward/backward."""

import pytest
import torch
import torch.nn.functional as F

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = a.detach().float(), b.detach().float()
    return float((a - b).norm() / b.norm().clamp_min(1e-12))


@pytest.mark.parametrize("B,H,Cin,Cout,stride", [(3, 20, 2, 32, 2), (2, 12, 32, 64, 1),
                                                 (4, 9, 16, 8, 2)])
def test_conv2d_layer(B, H, Cin, Cout, stride):
    from dgc_b200.warmstart import _Conv2d, _round8

    g = torch.Generator(device="cuda").manual_seed(B * 100 + Cin)
    x = torch.randn(B, H, H, Cin, device="cuda", generator=g).to(torch.bfloat16)
    K = 9 * Cin
    w = torch.zeros(Cout, _round8(K), device="cuda")
    w[:, :K] = torch.randn(Cout, K, device="cuda", generator=g) * 0.2
    w = w.to(torch.bfloat16).float().requires_grad_()
    b = (torch.randn(Cout, device="cuda", generator=g) * 0.1).requires_grad_()
    xin = x.clone().requires_grad_()
    y = _Conv2d.apply(xin, w, b, 3, stride, 1, True)
    # torch reference: weight [Cout, ky, kx, Cin] -> [Cout, Cin, ky, kx]
    wt = w[:, :K].detach().view(Cout, 3, 3, Cin).permute(0, 3, 1, 2).contiguous().requires_grad_()
    bt = b.detach().clone().requires_grad_()
    xt = x.float().permute(0, 3, 1, 2).contiguous().requires_grad_()
    yt = torch.relu(F.conv2d(xt, wt, bt, stride=stride, padding=1)).permute(0, 2, 3, 1)
    assert rel(y, yt) < 1e-2
    gy = torch.randn(yt.shape, device="cuda", generator=g).to(torch.bfloat16)
    gx, gw, gb = torch.autograd.grad(y, [xin, w, b], grad_outputs=gy)
    gxt, gwt, gbt = torch.autograd.grad(yt, [xt, wt, bt], grad_outputs=gy.float())
    assert rel(gw[:, :K].view(Cout, 3, 3, Cin).permute(0, 3, 1, 2), gwt) < 2e-2
    assert torch.count_nonzero(gw[:, K:]) == 0
    assert rel(gb, gbt) < 2e-2
    assert rel(gx, gxt.permute(0, 2, 3, 1)) < 2e-2


def test_view_conv_and_network():
    from dgc_b200.warmstart import WarmStartNet, _ViewConv

    g = torch.Generator(device="cuda").manual_seed(1)
    A, Cin, Cout, k = 37, 64, 24, 5
    f = torch.randn(A, Cin, device="cuda", generator=g).to(torch.bfloat16).requires_grad_()
    w = (torch.randn(Cout, k * Cin, device="cuda", generator=g) * 0.1).to(torch.bfloat16).float()
    w.requires_grad_()
    b = torch.zeros(Cout, device="cuda", requires_grad=True)
    y = _ViewConv.apply(f, w, b, k, False)
    # reference: circular conv1d over the view axis
    ft = f.detach().float().t()[None].requires_grad_()        # [1, Cin, A]
    wt = w.detach().view(Cout, k, Cin).permute(0, 2, 1).contiguous().requires_grad_()
    yt = F.conv1d(F.pad(ft, (k // 2, k // 2), mode="circular"), wt)[0].t()
    assert rel(y, yt) < 1e-2
    gy = torch.randn(A, Cout, device="cuda", generator=g)
    gf, gw = torch.autograd.grad(y, [f, w], grad_outputs=gy)
    gft, gwt = torch.autograd.grad(yt, [ft, wt], grad_outputs=gy)
    assert rel(gf, gft[0].t()) < 2e-2
    assert rel(gw.view(Cout, k, Cin).permute(0, 2, 1), gwt) < 2e-2

    net = WarmStartNet().cuda()
    assert 1.2e6 < sum(p.numel() for p in net.parameters()) < 2.5e6
    x = torch.randn(12, 96, 96, 2, device="cuda").to(torch.bfloat16)
    out = net(x)
    assert out.shape == (12, 8) and torch.isfinite(out).all()
    out.square().sum().backward()
    assert all(p.grad is not None and torch.isfinite(p.grad).all() for p in net.parameters())
