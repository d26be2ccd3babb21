"""Tensor-core (tcgen05) kernels of the learned preconditioner against plain
PyTorch FP32 references of the same ops on BF16-rounded inputs (GPU)."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


@pytest.fixture(scope="module")
def env():
    import torch
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    torch.manual_seed(0)
    return torch, nn, nn.Ops(dev), dev


def _rel(a, b):
    a, b = a.detach().double(), b.detach().double()
    return float((a.detach() - b.detach()).norm() / b.detach().norm())


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 48, 200), (1000, 128, 1152), (257, 100, 8),
                                   (2048, 64, 576)])
def test_gemm_matches_fp32_matmul(env, M, N, K):
    torch, nn, ops, dev = env
    a = torch.randn(M, K, device=dev).bfloat16()
    b = torch.randn(N, K, device=dev).bfloat16()
    d = torch.zeros(M, N, device=dev)
    ops.gemm(a, b, d)
    ref = a.float() @ b.float().t()
    torch.cuda.synchronize()
    assert int(ops.err.item()) == 0
    assert _rel(d, ref) < 1e-5, _rel(d, ref)


def _nchw(t):
    return t.permute(0, 3, 1, 2)


# widths that are multiples of 128 with 16-channel groups run the row kernel (taps as
# shifted operand windows), the others the implicit-im2col GEMM; (8, 16, 3, 128)
# runs the forward on the GEMM (8 input channels) and the input gradient on the row kernel
@pytest.mark.parametrize("ci,co,h,w", [(8, 16, 16, 24), (32, 64, 8, 8), (16, 128, 20, 12),
                                       (16, 16, 4, 128), (32, 64, 3, 256), (128, 64, 2, 128),
                                       (16, 128, 2, 128), (8, 16, 3, 128), (64, 32, 2, 384)])
def test_conv3x3_forward_and_gradients(env, ci, co, h, w):
    torch, nn, ops, dev = env
    F = torch.nn.functional
    n = 2
    x = torch.randn(n, h, w, ci, device=dev).bfloat16()
    wt = (torch.randn(co, 9 * ci, device=dev) * 0.1).bfloat16()
    bias = torch.randn(co, device=dev)
    y = torch.zeros(n, h, w, co, device=dev, dtype=torch.bfloat16)
    ops.conv(nn.act(x, n, h, w), wt, bias, nn.act(y, n, h, w), relu=True)
    w4 = wt.float().view(co, 3, 3, ci).permute(0, 3, 1, 2)      # [co][ci][ky][kx]
    xr = _nchw(x.float()).requires_grad_(True)
    w4r = w4.clone().requires_grad_(True)
    ref = F.relu(F.conv2d(xr, w4r, bias, padding=1))
    assert _rel(_nchw(y.float()), ref) < 1e-2
    # gradients through the pre-activation (a plain conv) with an upstream dy
    dy = torch.randn(n, h, w, co, device=dev).bfloat16()
    pre = F.conv2d(xr, w4r, None, padding=1)
    pre.backward(_nchw(dy.float()))
    wf = torch.zeros(ci, 9 * co, device=dev, dtype=torch.bfloat16)
    ops.flip3(wt, wf, co, ci)
    dx = torch.zeros(n, h, w, ci, device=dev, dtype=torch.bfloat16)
    ops.conv_dgrad(nn.act(dy, n, h, w), wf, nn.act(dx, n, h, w))
    dw = torch.zeros(co, 9 * ci, device=dev)
    ops.conv_wgrad(nn.act(x, n, h, w), nn.act(dy, n, h, w), dw)
    db = torch.zeros(co, device=dev)
    ops.bias_grad(nn.act(dy, n, h, w), db)
    torch.cuda.synchronize()
    assert int(ops.err.item()) == 0
    assert _rel(_nchw(dx.float()), xr.grad) < 1e-2
    assert _rel(dw.view(co, 3, 3, ci).permute(0, 3, 1, 2), w4r.grad) < 1e-3
    assert _rel(db, dy.float().sum(dim=(0, 1, 2))) < 1e-4


@pytest.mark.parametrize("ci,co,h,w", [(16, 8, 4, 6), (128, 64, 8, 8)])
def test_up2_forward_and_gradients(env, ci, co, h, w):
    torch, nn, ops, dev = env
    F = torch.nn.functional
    n = 2
    x = torch.randn(n, h, w, ci, device=dev).bfloat16()
    u = (torch.randn(4 * co, ci, device=dev) * 0.1).bfloat16()      # [(a*2+b)*co + o][c]
    bias = torch.randn(co, device=dev)
    y = torch.zeros(n, 2 * h, 2 * w, co, device=dev, dtype=torch.bfloat16)
    ops.up(nn.act(x, n, h, w), u, bias, nn.act(y, n, 2 * h, 2 * w), relu=False)
    # conv_transpose2d weight [ci][co][a][b]
    wt = u.float().view(2, 2, co, ci).permute(3, 2, 0, 1).contiguous().requires_grad_(True)
    xr = _nchw(x.float()).requires_grad_(True)
    ref = F.conv_transpose2d(xr, wt, bias, stride=2)
    assert _rel(_nchw(y.float()), ref) < 1e-2
    dy = torch.randn(n, 2 * h, 2 * w, co, device=dev).bfloat16()
    ref.backward(_nchw(dy.float()))
    ut = torch.zeros(ci, 4 * co, device=dev, dtype=torch.bfloat16)
    ops.transpose(u, ut, 4 * co, ci)
    dx = torch.zeros(n, h, w, ci, device=dev, dtype=torch.bfloat16)
    ops.up_dgrad(nn.act(dy, n, 2 * h, 2 * w), ut, nn.act(dx, n, h, w))
    du = torch.zeros(4 * co, ci, device=dev)
    ops.up_wgrad(nn.act(x, n, h, w), nn.act(dy, n, 2 * h, 2 * w), du)
    torch.cuda.synchronize()
    assert _rel(_nchw(dx.float()), xr.grad) < 1e-2
    assert _rel(du.view(2, 2, co, ci).permute(3, 2, 0, 1), wt.grad) < 1e-3


def test_pool_forward_and_backward(env):
    torch, nn, ops, dev = env
    F = torch.nn.functional
    n, h, w, c = 2, 8, 12, 16
    x = torch.randn(n, h, w, c, device=dev).bfloat16()
    y = torch.zeros(n, h // 2, w // 2, c, device=dev, dtype=torch.bfloat16)
    ops.pool(nn.act(x, n, h, w), y)
    xr = _nchw(x.float()).requires_grad_(True)
    ref = F.max_pool2d(xr, 2)
    assert torch.equal(_nchw(y.float()), ref)
    dy = torch.randn(n, h // 2, w // 2, c, device=dev).bfloat16()
    ref.backward(_nchw(dy.float()))
    dx = torch.zeros_like(x)
    ops.pool_bwd(nn.act(x, n, h, w), dy, nn.act(dx, n, h, w), relu_mask=False)
    torch.cuda.synchronize()
    assert torch.equal(_nchw(dx.float()), xr.grad)
