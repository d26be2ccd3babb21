"""The U-Net's tensor-core kernels against the FP64 CPU oracle (GPU).

The library's network (nn.py on the tcgen05 kernels of csrc/nn.cu) and its FP64
restatement (oracle/unet_oracle.py) with the same weights; the oracle rounds to
BF16 wherever the kernels store BF16 (weights, activations, intermediate
gradients).

Layer by layer (the strict check): every stored activation and gradient buffer
is recomputed by the oracle from the values the kernels stored for its operands
(`Net.replay`), so what remains is FP32 against FP64 accumulation followed by one
BF16 rounding: each element within one BF16 unit (2^-7 of its magnitude) plus
1e-5 of the buffer's largest value, pooling and the input cast exact, the FP32
output and every weight and bias gradient (FP32 accumulation of the stored BF16
operands) to relative L2 1e-4, the loss to 1e-5.

Whole network (a sanity bound): run from the input alone, a BF16 rounding that
lands on the other side of a tie in one layer carries into the next; over the
15 layers the output differs by 3.9e-3 relative L2 (measured), so the bounds
there are 1e-2 on the output and the loss and 5e-2 on the gradients.
"""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _one_unit(got, want, name):
    d = np.abs(got - want)
    allowed = 2.0 ** -7 * np.maximum(np.abs(got), np.abs(want)) + 1e-5 * np.abs(want).max()
    assert not (d > allowed).any(), (name, int((d > allowed).sum()), float(d.max()))
    assert _rel(got, want) < 3e-3, (name, _rel(got, want))


def _half(buf, key, c):
    if key.endswith("_enc"):
        return buf[key[:-4]][..., c:]
    if key.endswith("_up"):
        return buf[key[:-3]][..., :c]
    return buf[key]


def _setup(shape=(2, 32, 48)):
    import torch
    nn = importlib.import_module(PKG + ".nn")
    dev = torch.device("cuda", 0)
    net = nn.UNet(dev, seed=5)
    g = torch.Generator(device="cpu").manual_seed(6)
    x = torch.randn(*shape, 3, generator=g)
    target = torch.randn(*shape, 3, generator=g)
    loss = float(net.loss_grad(x.to(dev), target.to(dev)))
    torch.cuda.synchronize()
    assert int(net.ops.err.item()) == 0
    Bt, Gt = net.bufs[tuple(shape)]
    B = {k: _np(v) for k, v in Bt.items()}
    G = {k: _np(v) for k, v in Gt.items()}
    params = {k: (p.w.cpu().numpy(), p.b.cpu().numpy()) for k, p in net.params.items()}
    mine = {k: (p.g.cpu().numpy().astype(np.float64), p.bg.cpu().numpy().astype(np.float64))
            for k, p in net.params.items()}
    return net, x.numpy().astype(np.float64), target.numpy().astype(np.float64), loss, B, G, params, mine


# (1, 16, 256): levels 0 and 1 (widths 256, 128) run their 3x3 convolutions on
# the row kernel, the rest on the implicit-im2col GEMM
@pytest.mark.parametrize("shape", [(2, 32, 48), (1, 16, 256)])
def test_unet_layers_match_the_fp64_oracle(shape):
    import unet_oracle as U
    net, x, target, loss, B, G, params, mine = _setup(shape)
    ref = U.Net(params, bf16=True)
    xin = np.zeros(B["in0"].shape)
    xin[..., :U.IN_C] = x
    assert np.array_equal(B["in0"], U.to_bf16(xin))
    A, Gr, W = ref.replay(B, G, target)
    for k, v in A.items():
        c = U.LEVELS[int(k[3])] if k.startswith("cat") else 0
        got = _half(B, k, c)
        if k == "out":
            assert _rel(got, v) < 1e-4, (k, _rel(got, v))
        elif k.startswith("in"):
            assert np.array_equal(got, v), k
        else:
            _one_unit(got, v, k)
    for k, v in Gr.items():
        c = U.LEVELS[int(k[3])] if k.startswith("cat") else 0
        _one_unit(_half(G, k, c), v, "grad " + k)
    assert {"e0a", "e3b", "cat0_enc", "cat2_up", "in3", "d0b", "out"} <= set(A)
    assert set(W) == set(mine)
    for k, (rw, rb) in W.items():
        gw, gb = mine[k]
        assert _rel(gw, rw) < 1e-4 and _rel(gb, rb) < 1e-4, (k, _rel(gw, rw), _rel(gb, rb))
    n, h, w, _ = B["out"].shape
    d = B["out"][..., :U.OUT_C] - target
    ref_loss = float(np.sum(d ** 2) / (n * h * w * U.OUT_C))
    assert abs(loss - ref_loss) < 1e-5 * ref_loss, (loss, ref_loss)


def test_unet_whole_network_matches_the_fp64_oracle():
    import unet_oracle as U
    net, x, target, loss, B, G, params, mine = _setup()
    ref_out, ref_loss, grads = U.Net(params, bf16=True).loss_grad(x, target)
    out = B["out"][..., :U.OUT_C]
    assert _rel(out, ref_out) < 1e-2, _rel(out, ref_out)
    assert abs(loss - ref_loss) < 1e-2 * ref_loss, (loss, ref_loss)
    a, b = [], []
    report = {}
    for name, (gw, gb) in mine.items():
        rw, rb = grads[name]
        report[name] = (_rel(gw, rw), _rel(gb, rb))
        a += [gw.ravel(), gb]
        b += [rw.ravel(), rb]
    print("whole network, per-layer relative L2 (weights, biases):", report)
    assert _rel(np.concatenate(a), np.concatenate(b)) < 5e-2
