"""The U-Net's tensor-core kernels against the FP64 CPU oracle (GPU).

The library's network (nn.py on the tcgen05 kernels of csrc/nn.cu) and its FP64
restatement (oracle/unet_oracle.py) with the same weights: the oracle rounds to
BF16 wherever the kernels store BF16 (weights, activations, intermediate
gradients), so what remains between them is FP32 against FP64 accumulation and
the rare BF16 rounding that lands on the other side of a tie.  Checked: the
network output, the loss, and the weight and bias gradients of every layer.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_unet_gradients_match_the_fp64_oracle():
    import torch
    import unet_oracle as U
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    net = nn.UNet(dev, seed=5)
    g = torch.Generator(device="cpu").manual_seed(6)
    x = torch.randn(2, 32, 48, 3, generator=g)
    target = torch.randn(2, 32, 48, 3, generator=g)
    loss = float(net.loss_grad(x.to(dev), target.to(dev)))
    out = net.bufs[(2, 32, 48)][0]["out"][..., :3].float().cpu().numpy()
    torch.cuda.synchronize()
    assert int(net.ops.err.item()) == 0
    params = {k: (p.w.cpu().numpy(), p.b.cpu().numpy()) for k, p in net.params.items()}
    ref_out, ref_loss, grads = U.Net(params, bf16=True).loss_grad(x.numpy().astype(np.float64),
                                                                    target.numpy().astype(np.float64))
    assert _rel(out, ref_out) < 1e-3, _rel(out, ref_out)
    assert abs(loss - ref_loss) < 1e-3 * ref_loss, (loss, ref_loss)
    report = {}
    mine, theirs = [], []
    for name, p in net.params.items():
        gw, gb = p.g.cpu().numpy(), p.bg.cpu().numpy()
        rw, rb = grads[name]
        report[name] = (_rel(gw, rw), _rel(gb, rb))
        mine += [gw.ravel(), gb]
        theirs += [rw.ravel(), rb]
    print("per-layer relative L2 (weights, biases):", report)
    bad = {k: v for k, v in report.items() if not (v[0] < 2e-2 and v[1] < 2e-2)}
    assert not bad, bad
    assert _rel(np.concatenate(mine), np.concatenate(theirs)) < 5e-3
