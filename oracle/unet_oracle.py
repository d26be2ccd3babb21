"""FP64 CPU restatement of the learned preconditioner's U-Net — TEST INFRASTRUCTURE ONLY.

Forward pass, mean-squared-error loss and the full backward pass (weight, bias
and input gradients) of the network that nn.py builds on the library's tensor-core
kernels, in float64 numpy.  Only tests/ import it, to check the kernels'
gradients.  The reference has no learned component; this restates the
library's own network:

  * 4 levels of two 3x3 convolutions (pad 1) + ReLU with 16-32-64-128 channels,
    2x2 max pooling down (the gradient goes to the first maximum of a window in
    row-major order, and only where that maximum is positive, as the ReLU before
    it), 2x2 stride-2 transposed convolutions + ReLU up, skip connections by
    channel concatenation [up | encoder], a final 3x3 convolution without ReLU;
  * input 3 channels padded to 8, output 16 channels of which the first 3 count;
  * weights as the library stores them: a convolution [co][tap * ci + c] with
    tap = ky * 3 + kx, a transposed convolution [(a * 2 + b) * co + o][c];
  * loss = mean over the first 3 output channels of (y - t)^2.

With `bf16=True` every value the kernels store in BF16 (weights, activations,
intermediate gradients, the loss gradient) is rounded to BF16 at the same point
(round to nearest even); sums and products stay float64.  With `bf16=False` it
is the exact float64 network (for finite-difference checks of this file).
Arrays are NHWC float64.

`loss_grad` runs the whole network from the input; `replay` recomputes every
layer from the values the kernels stored for its operands (buffer names of
nn.py), so that a BF16 rounding which lands on the other side of a tie in one
layer does not carry into the next and each layer can be checked to one BF16
unit.
"""
from __future__ import annotations

import numpy as np

LEVELS = (16, 32, 64, 128)
IN_C, IN_P, OUT_C, OUT_P = 3, 8, 3, 16


def to_bf16(x):
    """Round to the nearest BF16 value (ties to even), through float32."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


class Net:
    """params: name -> (w, b) float64, w in the library's layout (see module docstring)."""

    def __init__(self, params: dict, bf16: bool = True):
        self.P = {k: (np.asarray(w, np.float64), np.asarray(b, np.float64)) for k, (w, b) in params.items()}
        self.bf16 = bf16
        self.r = to_bf16 if bf16 else (lambda a: a)

    # ---- building blocks ------------------------------------------------------
    @staticmethod
    def _patches(x):
        """3x3, pad-1 im2col: (n, h, w, c) -> (n, h, w, 9 c), tap-major."""
        n, h, w, c = x.shape
        xp = np.zeros((n, h + 2, w + 2, c))
        xp[:, 1:-1, 1:-1] = x
        cols = [xp[:, ky:ky + h, kx:kx + w] for ky in range(3) for kx in range(3)]
        return np.concatenate(cols, axis=3)

    def _conv(self, x, w, b):
        return self._patches(x) @ w.T + b

    def _conv_dx(self, g, w, ci):
        """input gradient of a 3x3 convolution: g (n, h, w, co) -> (n, h, w, ci)"""
        n, h, wd, co = g.shape
        wt = w.reshape(co, 9, ci)
        gp = np.zeros((n, h + 2, wd + 2, co))
        gp[:, 1:-1, 1:-1] = g
        dx = np.zeros((n, h, wd, ci))
        for ky in range(3):
            for kx in range(3):
                # output pixel p reads x at p + (ky - 1, kx - 1): x pixel q gets g at q - shift
                gs = gp[:, 2 - ky:2 - ky + h, 2 - kx:2 - kx + wd]
                dx += gs @ wt[:, ky * 3 + kx, :]
        return dx

    def _conv_dw(self, x, g):
        n, h, w, co = g.shape
        pa = self._patches(x).reshape(-1, 9 * x.shape[3])
        return g.reshape(-1, co).T @ pa, g.reshape(-1, co).sum(0)

    @staticmethod
    def _up(x, w, b, co):
        n, h, wd, ci = x.shape
        y = np.zeros((n, 2 * h, 2 * wd, co))
        for a in range(2):
            for bb in range(2):
                ab = a * 2 + bb
                y[:, a::2, bb::2] = x @ w[ab * co:(ab + 1) * co].T + b
        return y

    @staticmethod
    def _up_dx(g, w, co, ci):
        n, H, W, _ = g.shape
        dx = np.zeros((n, H // 2, W // 2, ci))
        for a in range(2):
            for bb in range(2):
                ab = a * 2 + bb
                dx += g[:, a::2, bb::2] @ w[ab * co:(ab + 1) * co]
        return dx

    @staticmethod
    def _up_dw(x, g, co):
        ci = x.shape[3]
        dw = np.zeros((4 * co, ci))
        for a in range(2):
            for bb in range(2):
                ab = a * 2 + bb
                dw[ab * co:(ab + 1) * co] = g[:, a::2, bb::2].reshape(-1, co).T @ x.reshape(-1, ci)
        return dw, g.reshape(-1, co).sum(0)

    @staticmethod
    def _pool(x):
        n, h, w, c = x.shape
        v = x.reshape(n, h // 2, 2, w // 2, 2, c)
        return v.max(axis=(2, 4))

    @staticmethod
    def _pool_back(x, gy):
        """gradient to the first maximum (row-major in the 2x2 window) where it is > 0"""
        n, h, w, c = x.shape
        v = x.reshape(n, h // 2, 2, w // 2, 2, c).transpose(0, 1, 3, 5, 2, 4).reshape(n, h // 2, w // 2, c, 4)
        first = np.argmax(v, axis=4)                   # first occurrence of the maximum
        m = np.take_along_axis(v, first[..., None], axis=4)[..., 0]
        g = np.where(m > 0, gy, 0.0)
        out = np.zeros((n, h // 2, w // 2, c, 4))
        np.put_along_axis(out, first[..., None], g[..., None], axis=4)
        return out.reshape(n, h // 2, w // 2, c, 2, 2).transpose(0, 1, 4, 2, 5, 3).reshape(n, h, w, c)

    def _W(self, name):
        w, b = self.P[name]
        return self.r(w), b

    # ---- forward / loss / backward -------------------------------------------
    def loss_grad(self, x, target):
        """x, target: (n, h, w, 3).  Returns (output (n, h, w, 3), loss, grads name -> (dw, db)).
        The stored activations and gradients are kept in `self.stored` as (B, G)
        under the buffer names of nn.py (the input of `replay`)."""
        r = self.r
        n, h, w, _ = x.shape
        relu = lambda a: np.maximum(a, 0.0)
        A = {}
        xin = np.zeros((n, h, w, IN_P))
        xin[..., :IN_C] = x
        cur = r(xin)
        for l, c in enumerate(LEVELS):
            A[f"in{l}"] = cur
            wa, ba = self._W(f"e{l}a")
            A[f"e{l}a"] = r(relu(self._conv(cur, wa, ba)))
            wb, bb = self._W(f"e{l}b")
            A[f"e{l}b"] = r(relu(self._conv(A[f"e{l}a"], wb, bb)))
            if l < 3:
                cur = self._pool(A[f"e{l}b"])
        prev = A["e3b"]
        for l in (2, 1, 0):
            c = LEVELS[l]
            wu, bu = self._W(f"u{l}")
            up = r(relu(self._up(prev, wu, bu, c)))
            A[f"cat{l}"] = np.concatenate([up, A[f"e{l}b"]], axis=3)
            wa, ba = self._W(f"d{l}a")
            A[f"d{l}a"] = r(relu(self._conv(A[f"cat{l}"], wa, ba)))
            wb, bb = self._W(f"d{l}b")
            A[f"d{l}b"] = r(relu(self._conv(A[f"d{l}a"], wb, bb)))
            prev = A[f"d{l}b"]
        wo, bo = self._W("out")
        y = self._conv(prev, wo, bo)                  # float output, no ReLU
        cnt = n * h * w * OUT_C
        d = np.zeros_like(y)
        d[..., :OUT_C] = y[..., :OUT_C] - target
        loss = float(np.sum(d ** 2) / cnt)
        gout = r(2.0 / cnt * d)

        G = {}
        grads = {}
        SG = {"out": gout}
        grads["out"] = self._conv_dw(A["d0b"], gout)
        g = r(self._conv_dx(gout, wo, LEVELS[0]) * (A["d0b"] > 0))
        SG["d0b"] = g
        for l in (0, 1, 2):
            c = LEVELS[l]
            wb, _ = self._W(f"d{l}b")
            grads[f"d{l}b"] = self._conv_dw(A[f"d{l}a"], g)
            g = r(self._conv_dx(g, wb, c) * (A[f"d{l}a"] > 0))
            SG[f"d{l}a"] = g
            wa, _ = self._W(f"d{l}a")
            grads[f"d{l}a"] = self._conv_dw(A[f"cat{l}"], g)
            gcat = r(self._conv_dx(g, wa, 2 * c) * (A[f"cat{l}"] > 0))
            G[f"cat{l}"] = gcat
            gup = gcat[..., :c]
            src = A["e3b"] if l == 2 else A[f"d{l + 1}b"]
            wu, _ = self._W(f"u{l}")
            grads[f"u{l}"] = self._up_dw(src, gup, c)
            g = r(self._up_dx(gup, wu, c, src.shape[3]) * (src > 0))
            SG["e3b" if l == 2 else f"d{l + 1}b"] = g
        # g is now the gradient at e3b
        for l in (3, 2, 1, 0):
            c = LEVELS[l]
            if l == 3:
                geb = g
            else:
                # the skip gradient (from cat) plus the pooled path, summed in BF16 storage
                geb = r(G[f"cat{l}"][..., c:] + self._pool_back(A[f"e{l}b"], gin))
                SG[f"cat{l}"] = np.concatenate([G[f"cat{l}"][..., :c], geb], axis=3)
            wb, _ = self._W(f"e{l}b")
            grads[f"e{l}b"] = self._conv_dw(A[f"e{l}a"], geb)
            gea = r(self._conv_dx(geb, wb, c) * (A[f"e{l}a"] > 0))
            SG[f"e{l}a"] = gea
            wa, _ = self._W(f"e{l}a")
            grads[f"e{l}a"] = self._conv_dw(A[f"in{l}"], gea)
            if l > 0:
                gin = r(self._conv_dx(gea, wa, A[f"in{l}"].shape[3]))
                SG[f"in{l}"] = gin
        SB = {k: v for k, v in A.items() if not (k.startswith("e") and k.endswith("b") and k != "e3b")}
        SB["out"] = y
        self.stored = (SB, SG)
        return y[..., :OUT_C], loss, grads

    # ---- layer-by-layer replay --------------------------------------------
    def replay(self, B, G, target):
        """B, G: the kernels' stored activation and gradient buffers (nn.py names; the
        BF16 values as float64; B["out"] the FP32 output), target (n, h, w, 3).
        Returns (acts, grads, wgrads): the value of every stored buffer recomputed
        from the stored values it is made of (the encoder half of cat{l} under
        "cat{l}_enc", the up-sampled half under "cat{l}_up"), and the weight and
        bias gradients of every layer from the stored operands."""
        r = self.r
        relu = lambda a: np.maximum(a, 0.0)
        A, Gr, W = {}, {}, {}
        for l, c in enumerate(LEVELS):
            wa, ba = self._W(f"e{l}a")
            wb, bb = self._W(f"e{l}b")
            A[f"e{l}a"] = r(relu(self._conv(B[f"in{l}"], wa, ba)))
            eb = r(relu(self._conv(B[f"e{l}a"], wb, bb)))
            if l < 3:
                A[f"cat{l}_enc"] = eb
                A[f"in{l + 1}"] = self._pool(B[f"cat{l}"][..., c:])
            else:
                A["e3b"] = eb
        for l in (2, 1, 0):
            c = LEVELS[l]
            src = B["e3b"] if l == 2 else B[f"d{l + 1}b"]
            wu, bu = self._W(f"u{l}")
            A[f"cat{l}_up"] = r(relu(self._up(src, wu, bu, c)))
            wa, ba = self._W(f"d{l}a")
            A[f"d{l}a"] = r(relu(self._conv(B[f"cat{l}"], wa, ba)))
            wb, bb = self._W(f"d{l}b")
            A[f"d{l}b"] = r(relu(self._conv(B[f"d{l}a"], wb, bb)))
        wo, bo = self._W("out")
        A["out"] = self._conv(B["d0b"], wo, bo)

        y = B["out"]
        n, h, w, _ = y.shape
        cnt = n * h * w * OUT_C
        d = np.zeros_like(y)
        d[..., :OUT_C] = y[..., :OUT_C] - target
        Gr["out"] = r(2.0 / cnt * d)
        W["out"] = self._conv_dw(B["d0b"], G["out"])
        Gr["d0b"] = r(self._conv_dx(G["out"], wo, LEVELS[0]) * (B["d0b"] > 0))
        skip = {}
        for l in (0, 1, 2):
            c = LEVELS[l]
            wb, _ = self._W(f"d{l}b")
            W[f"d{l}b"] = self._conv_dw(B[f"d{l}a"], G[f"d{l}b"])
            Gr[f"d{l}a"] = r(self._conv_dx(G[f"d{l}b"], wb, c) * (B[f"d{l}a"] > 0))
            wa, _ = self._W(f"d{l}a")
            W[f"d{l}a"] = self._conv_dw(B[f"cat{l}"], G[f"d{l}a"])
            gcat = r(self._conv_dx(G[f"d{l}a"], wa, 2 * c) * (B[f"cat{l}"] > 0))
            Gr[f"cat{l}_up"] = gcat[..., :c]
            skip[l] = gcat[..., c:]
            sname = "e3b" if l == 2 else f"d{l + 1}b"
            src = B[sname]
            wu, _ = self._W(f"u{l}")
            gup = G[f"cat{l}"][..., :c]
            W[f"u{l}"] = self._up_dw(src, gup, c)
            Gr[sname] = r(self._up_dx(gup, wu, c, src.shape[3]) * (src > 0))
        for l in (3, 2, 1, 0):
            c = LEVELS[l]
            if l == 3:
                geb = G["e3b"]
            else:
                Gr[f"cat{l}_enc"] = r(skip[l] + self._pool_back(B[f"cat{l}"][..., c:], G[f"in{l + 1}"]))
                geb = G[f"cat{l}"][..., c:]
            wb, _ = self._W(f"e{l}b")
            W[f"e{l}b"] = self._conv_dw(B[f"e{l}a"], geb)
            Gr[f"e{l}a"] = r(self._conv_dx(geb, wb, c) * (B[f"e{l}a"] > 0))
            wa, _ = self._W(f"e{l}a")
            W[f"e{l}a"] = self._conv_dw(B[f"in{l}"], G[f"e{l}a"])
            if l > 0:
                Gr[f"in{l}"] = r(self._conv_dx(G[f"e{l}a"], wa, B[f"in{l}"].shape[3]))
        return A, Gr, W
