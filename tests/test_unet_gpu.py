"""The U-Net on the tensor-core kernels: its loss gradient against PyTorch autograd
of the same network (BF16-rounded like the kernels' storage), and Adam training
lowering the loss (GPU)."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def _torch_reference(torch, net, x, nn):
    F = torch.nn.functional
    r = lambda t: t.bfloat16().float()
    P = net.params
    leaves = {}

    def W(name):
        p = P[name]
        if p.kind == "conv":
            w = p.wb.float().view(p.co, 3, 3, p.ci).permute(0, 3, 1, 2).contiguous()
        else:
            w = p.wb.float().view(2, 2, p.co, p.ci).permute(3, 2, 0, 1).contiguous()
        w.requires_grad_(True)
        b = p.b.clone().requires_grad_(True)
        leaves[name] = (w, b)
        return w, b

    n, h, wd, _ = x.shape
    xin = torch.zeros(n, nn.IN_P, h, wd, device=x.device)
    xin[:, :3] = x.permute(0, 3, 1, 2)
    hcur, skips = r(xin), []
    for l in range(4):
        w, b = W(f"e{l}a")
        a = r(F.relu(F.conv2d(hcur, w, b, padding=1)))
        w, b = W(f"e{l}b")
        e = r(F.relu(F.conv2d(a, w, b, padding=1)))
        if l < 3:
            skips.append(e)
            hcur = F.max_pool2d(e, 2)
        else:
            hcur = e
    for l in (2, 1, 0):
        w, b = W(f"u{l}")
        u = r(F.relu(F.conv_transpose2d(hcur, w, b, stride=2)))
        cat = torch.cat([u, skips[l]], 1)
        w, b = W(f"d{l}a")
        a = r(F.relu(F.conv2d(cat, w, b, padding=1)))
        w, b = W(f"d{l}b")
        hcur = r(F.relu(F.conv2d(a, w, b, padding=1)))
    w, b = W("out")
    out = F.conv2d(hcur, w, b, padding=1)
    return out[:, :3].permute(0, 2, 3, 1), leaves


def test_unet_loss_gradient_matches_autograd():
    import torch
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    net = nn.UNet(dev, seed=1)
    g = torch.Generator(device="cpu").manual_seed(2)
    x = torch.randn(2, 32, 48, 3, generator=g).to(dev)
    target = torch.randn(2, 32, 48, 3, generator=g).to(dev)
    loss = net.loss_grad(x, target)
    out = net.bufs[(2, 32, 48)][0]["out"][..., :3].clone()
    ref, leaves = _torch_reference(torch, net, x, nn)
    rl = torch.mean((ref - target) ** 2)
    rl.backward()
    torch.cuda.synchronize()
    assert int(net.ops.err.item()) == 0
    ref = ref.detach()
    assert float((out - ref).norm() / ref.norm()) < 3e-2
    assert abs(float(loss) - float(rl.detach())) < 2e-2 * float(rl.detach())
    # the kernels store every intermediate gradient in BF16 (autograd keeps FP32):
    # per-layer agreement degrades with depth into the backward pass, to ~10 %
    mine, theirs = [], []
    for name, (w, b) in leaves.items():
        p = net.params[name]
        if p.kind == "conv":
            gw = w.grad.permute(0, 2, 3, 1).reshape(p.co, 9 * p.ci)
        else:
            gw = w.grad.permute(2, 3, 1, 0).reshape(4 * p.co, p.ci)
        cos = float(torch.nn.functional.cosine_similarity(p.g.flatten(), gw.flatten(), dim=0))
        rel = float((p.g - gw).norm() / gw.norm().clamp_min(1e-30))
        assert cos > 0.98 and rel < 0.2, (name, cos, rel)
        relb = float((p.bg - b.grad).norm() / b.grad.norm().clamp_min(1e-30))
        assert relb < 0.2, (name, relb)
        mine += [p.g.flatten(), p.bg]
        theirs += [gw.flatten(), b.grad]
    cos = float(torch.nn.functional.cosine_similarity(torch.cat(mine), torch.cat(theirs), dim=0))
    assert cos > 0.995, cos


def test_unet_training_lowers_the_loss():
    import torch
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    net = nn.UNet(dev, seed=3)
    g = torch.Generator(device="cpu").manual_seed(4)
    x = torch.randn(4, 32, 64, 3, generator=g).to(dev)
    # a smooth, learnable target: a blurred, channel-mixed copy of the input
    k = torch.ones(3, 1, 5, 5, device=dev) / 25.0
    xb = torch.nn.functional.conv2d(x.permute(0, 3, 1, 2), k, padding=2, groups=3)
    target = (xb[:, [1, 2, 0]] * 2.0).permute(0, 2, 3, 1).contiguous()
    first = float(net.step(x, target, lr=2e-3))
    for _ in range(150):
        last = float(net.step(x, target, lr=2e-3))
    assert last < 0.3 * first, (first, last)
