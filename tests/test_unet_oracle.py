"""The FP64 U-Net oracle checked against its own finite differences (CPU).

oracle/unet_oracle.py restates the learned preconditioner's network (forward,
loss, backward) in float64; with BF16 rounding switched off it must be the exact
gradient of its own loss.  Centred differences on a few weights of every layer
and on the biases, at random points of a small input, pin it.
"""
import numpy as np
import pytest


def _params(rng, scale=1.0):
    import unet_oracle as U
    P = {}
    cin = U.IN_P
    for l, c in enumerate(U.LEVELS):
        P[f"e{l}a"] = (rng.standard_normal((c, 9 * cin)) * np.sqrt(2.0 / (9 * cin)), 0.1 * rng.standard_normal(c))
        P[f"e{l}b"] = (rng.standard_normal((c, 9 * c)) * np.sqrt(2.0 / (9 * c)), 0.1 * rng.standard_normal(c))
        cin = c
    for l in (2, 1, 0):
        c = U.LEVELS[l]
        P[f"u{l}"] = (rng.standard_normal((4 * c, U.LEVELS[l + 1])) * np.sqrt(2.0 / U.LEVELS[l + 1]),
                      0.1 * rng.standard_normal(c))
        P[f"d{l}a"] = (rng.standard_normal((c, 18 * c)) * np.sqrt(2.0 / (18 * c)), 0.1 * rng.standard_normal(c))
        P[f"d{l}b"] = (rng.standard_normal((c, 9 * c)) * np.sqrt(2.0 / (9 * c)), 0.1 * rng.standard_normal(c))
    P["out"] = (rng.standard_normal((U.OUT_P, 9 * 16)) * 0.1 * np.sqrt(2.0 / 144), 0.1 * rng.standard_normal(U.OUT_P))
    return P


@pytest.mark.parametrize("layer", ["e0a", "e1b", "e3a", "u2", "u0", "d1a", "d0b", "out"])
def test_oracle_gradient_is_the_derivative_of_its_loss(layer):
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import unet_oracle as U
    rng = np.random.default_rng(11)
    P = _params(rng)
    x = rng.standard_normal((1, 16, 24, 3))
    t = rng.standard_normal((1, 16, 24, 3))
    net = U.Net(P, bf16=False)
    _, _, grads = net.loss_grad(x, t)
    w, b = P[layer]
    h = 1e-6
    for _ in range(4):
        idx = tuple(rng.integers(0, s) for s in w.shape)
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        lp = U.Net({**P, layer: (wp, b)}, bf16=False).loss_grad(x, t)[1]
        lm = U.Net({**P, layer: (wm, b)}, bf16=False).loss_grad(x, t)[1]
        fd = (lp - lm) / (2 * h)
        an = grads[layer][0][idx]
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)) + 1e-7, (layer, idx, fd, an)
    q = int(rng.integers(0, b.shape[0]))
    bp, bm = b.copy(), b.copy()
    bp[q] += h
    bm[q] -= h
    fd = (U.Net({**P, layer: (w, bp)}, bf16=False).loss_grad(x, t)[1] -
          U.Net({**P, layer: (w, bm)}, bf16=False).loss_grad(x, t)[1]) / (2 * h)
    assert abs(fd - grads[layer][1][q]) <= 1e-6 * max(1.0, abs(fd)) + 1e-7


def test_bf16_rounding_matches_torch():
    import sys
    import os
    import torch
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import unet_oracle as U
    v = np.random.default_rng(3).standard_normal(10000) * 10.0 ** np.random.default_rng(4).integers(-20, 20, 10000)
    ref = torch.from_numpy(v.astype(np.float32)).bfloat16().float().numpy().astype(np.float64)
    assert np.array_equal(U.to_bf16(v), ref)


@pytest.mark.parametrize("bf16", [True, False])
def test_replay_reproduces_the_whole_network(bf16):
    """Fed the buffers the whole-network pass stored, the layer-by-layer replay
    recomputes every one of them and every weight gradient exactly."""
    import sys
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import unet_oracle as U
    rng = np.random.default_rng(12)
    P = _params(rng)
    x = rng.standard_normal((2, 16, 24, 3))
    t = rng.standard_normal((2, 16, 24, 3))
    net = U.Net(P, bf16=bf16)
    _, _, grads = net.loss_grad(x, t)
    B, G = net.stored
    A, Gr, W = net.replay(B, G, t)
    for k, v in A.items():
        if k.endswith("_enc"):
            want = B[k[:-4]][..., U.LEVELS[int(k[3])]:]
        elif k.endswith("_up"):
            want = B[k[:-3]][..., :U.LEVELS[int(k[3])]]
        else:
            want = B[k]
        assert np.array_equal(v, want), k
    for k, v in Gr.items():
        if k.endswith("_enc"):
            want = G[k[:-4]][..., U.LEVELS[int(k[3])]:]
        elif k.endswith("_up"):
            want = G[k[:-3]][..., :U.LEVELS[int(k[3])]]
        else:
            want = G[k]
        assert np.array_equal(v, want), k
    assert set(W) == set(grads)
    for k in W:
        assert np.array_equal(W[k][0], grads[k][0]) and np.array_equal(W[k][1], grads[k][1]), k
    names = {k.split("_")[0] for k in list(A) + list(Gr)}
    assert {"e0a", "e3b", "cat0", "cat2", "in3", "d0b", "out"} <= names
