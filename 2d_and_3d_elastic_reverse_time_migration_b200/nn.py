"""Learned LSRTM preconditioner: a 2D U-Net on the library's tensor-core kernels.

The network (4 levels, 16-32-64-128 channels, two 3x3 convolutions + ReLU per
level, 2x2 max pooling down, 2x2 stride-2 transposed convolutions + ReLU up,
skip connections by channel concatenation, a final 3x3 convolution) maps the
first LSRTM gradient (g_vp, g_vs, g_rho) to the reflectivity (r_vp, r_vs, r_rho)
that several CG iterations would reach.  Every convolution, its input and weight
gradients run on the hand-written tcgen05 kernels of csrc/nn.cu (BF16 activations
and weights, FP32 accumulation): an implicit-im2col GEMM, and for the 3x3
convolutions of layers at least 128 pixels wide a row kernel that reads the
nine taps from three staged input rows; pooling, bias gradients, the loss and
Adam are hand-written kernels too.  Torch only allocates the buffers (plumbing) and
calls nothing but the library on them.

Activations are NHWC BF16; channel counts are padded to multiples of 8 (input
3 -> 8, output 3 -> 16).  The reference has no learned component.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import ErtmError, _NnAct, lib

IN_C, OUT_C = 3, 3
IN_P, OUT_P = 8, 16
LEVELS = (16, 32, 64, 128)


def _ck(rc: int, what: str):
    if rc != 0:
        raise ErtmError(rc, what)


def act(t, n, h, w, c=None, off=0):
    """ertm_nn_act view of a BF16 NHWC tensor whose last dim is the channel stride."""
    cs = t.shape[-1]
    a = _NnAct()
    a.data, a.n, a.h, a.w = t.data_ptr(), n, h, w
    a.cstride, a.coff, a.c = cs, off, cs - off if c is None else c
    return a


def _p(t):
    return None if t is None else t.data_ptr()


class Ops:
    """Thin wrappers of the C ABI on CUDA tensors (stream = torch's current stream)."""

    def __init__(self, device):
        import torch
        self.torch = torch
        self.L = lib()
        self.dev = device
        self.err = torch.zeros(1, dtype=torch.int32, device=device)

    @property
    def st(self):
        return self.torch.cuda.current_stream(self.dev).cuda_stream

    def gemm(self, a, b, d):
        M, K = a.shape
        N = b.shape[0]
        _ck(self.L.ertm_nn_gemm(_p(a), _p(b), _p(d), M, N, K, _p(self.err), self.st), "gemm")

    def conv(self, x, w, bias, y, relu=True, y32=None):
        _ck(self.L.ertm_nn_conv3x3(C.byref(x), _p(w), _p(bias), C.byref(y), int(relu), _p(y32),
                                   _p(self.err), self.st), "conv3x3")

    def conv_dgrad(self, dy, wf, dx, mask=None):
        _ck(self.L.ertm_nn_conv3x3_dgrad(C.byref(dy), _p(wf), C.byref(dx),
                                         C.byref(mask) if mask is not None else None, _p(self.err),
                                         self.st), "conv3x3_dgrad")

    def conv_wgrad(self, x, dy, dw, splitk=0):
        P = x.n * x.h * x.w
        sk = splitk or max(1, min(148 * 2, P // 4096))
        _ck(self.L.ertm_nn_conv3x3_wgrad(C.byref(x), C.byref(dy), _p(dw), sk, _p(self.err), self.st),
            "conv3x3_wgrad")

    def up(self, x, u, bias, y, relu=True):
        _ck(self.L.ertm_nn_up2(C.byref(x), _p(u), _p(bias), C.byref(y), int(relu), _p(self.err),
                               self.st), "up2")

    def up_dgrad(self, dy, ut, dx, mask=None):
        _ck(self.L.ertm_nn_up2_dgrad(C.byref(dy), _p(ut), C.byref(dx),
                                     C.byref(mask) if mask is not None else None, _p(self.err),
                                     self.st), "up2_dgrad")

    def up_wgrad(self, x, dy, du, splitk=0):
        P = x.n * x.h * x.w
        sk = splitk or max(1, min(148 * 2, P // 4096))
        _ck(self.L.ertm_nn_up2_wgrad(C.byref(x), C.byref(dy), _p(du), sk, _p(self.err), self.st),
            "up2_wgrad")

    def pool(self, x, y):
        _ck(self.L.ertm_nn_pool2(C.byref(x), _p(y), self.st), "pool2")

    def pool_bwd(self, x, dy, dx, relu_mask=True):
        _ck(self.L.ertm_nn_pool2_bwd(C.byref(x), _p(dy), C.byref(dx), int(relu_mask), self.st),
            "pool2_bwd")

    def bias_grad(self, dy, db):
        _ck(self.L.ertm_nn_bias_grad(C.byref(dy), _p(db), self.st), "bias_grad")

    def mse(self, y32, target, c, scale, grad, loss):
        P = target.numel() // c
        _ck(self.L.ertm_nn_mse(_p(y32), _p(target), y32.shape[-1], c, P, scale, _p(grad), _p(loss),
                               self.st), "mse")

    def adam(self, w, g, m, v, wb, lr, step, b1=0.9, b2=0.999, eps=1e-8):
        _ck(self.L.ertm_nn_adam(_p(w), _p(g), _p(m), _p(v), _p(wb), w.numel(), lr, b1, b2, eps, step,
                                self.st), "adam")

    def flip3(self, w, wf, co, ci):
        _ck(self.L.ertm_nn_flip3(_p(w), _p(wf), co, ci, self.st), "flip3")

    def transpose(self, a, t, rows, cols):
        _ck(self.L.ertm_nn_transpose(_p(a), _p(t), rows, cols, self.st), "transpose")

    def to_bf16(self, a, b):
        _ck(self.L.ertm_nn_to_bf16(_p(a), _p(b), a.numel(), self.st), "to_bf16")


@dataclass
class Param:
    w: object      # FP32 master
    wb: object     # BF16 copy
    g: object      # FP32 gradient
    m: object
    v: object
    aux: object    # BF16 flipped / transposed copy for the input gradient
    kind: str      # "conv" or "up"
    co: int
    ci: int
    b: object      # FP32 bias
    bg: object
    bm: object
    bv: object
    bb: object     # unused BF16 slot of the bias (Adam writes one)


class UNet:
    """The 4-level U-Net; `forward`, `backward` and `step` run on the library kernels."""

    def __init__(self, device, seed: int = 0):
        import torch
        self.torch = torch
        self.dev = device
        self.ops = Ops(device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.params = {}
        cin = IN_P
        for l, c in enumerate(LEVELS):
            self._conv(f"e{l}a", cin, c, g)
            self._conv(f"e{l}b", c, c, g)
            cin = c
        for l in (2, 1, 0):
            c = LEVELS[l]
            self._up(f"u{l}", LEVELS[l + 1], c, g)
            self._conv(f"d{l}a", 2 * c, c, g)
            self._conv(f"d{l}b", c, c, g)
        self._conv("out", LEVELS[0], OUT_P, g, scale=0.1)
        self.t = 0
        self.bufs = {}
        self.refresh()

    # ---- parameters ---------------------------------------------------------
    def _new(self, shape, dtype=None):
        t = self.torch
        return t.zeros(shape, dtype=dtype or t.float32, device=self.dev)

    def _param(self, name, kind, co, ci, K, rows, g, scale=1.0):
        t = self.torch
        w = (t.randn((rows, K), generator=g) * (scale * (2.0 / K) ** 0.5)).to(self.dev)
        if kind == "conv" and ci == IN_P:                     # padded input channels carry nothing
            w.view(rows, 9, ci)[:, :, IN_C:] = 0
        bias_n = co
        p = Param(w=w, wb=self._new((rows, K), t.bfloat16), g=self._new((rows, K)), m=self._new((rows, K)),
                  v=self._new((rows, K)), aux=self._new((ci, (9 if kind == "conv" else 4) * co), t.bfloat16),
                  kind=kind, co=co, ci=ci, b=self._new(bias_n), bg=self._new(bias_n), bm=self._new(bias_n),
                  bv=self._new(bias_n), bb=self._new(bias_n, t.bfloat16))
        self.params[name] = p

    def _conv(self, name, ci, co, g, scale=1.0):
        self._param(name, "conv", co, ci, 9 * ci, co, g, scale)

    def _up(self, name, ci, co, g):
        self._param(name, "up", co, ci, ci, 4 * co, g)

    def refresh(self):
        """BF16 copies and the re-laid-out weights of the input gradients."""
        o = self.ops
        for p in self.params.values():
            o.to_bf16(p.w, p.wb)
            if p.kind == "conv":
                o.flip3(p.wb, p.aux, p.co, p.ci)
            else:
                o.transpose(p.wb, p.aux, 4 * p.co, p.ci)

    def state_dict(self):
        return {k: (p.w.cpu().numpy(), p.b.cpu().numpy()) for k, p in self.params.items()}

    def load_state_dict(self, sd):
        for k, (w, b) in sd.items():
            self.params[k].w.copy_(self.torch.from_numpy(w))
            self.params[k].b.copy_(self.torch.from_numpy(b))
        self.refresh()

    # ---- buffers ------------------------------------------------------------
    def _buffers(self, n, h, w):
        key = (n, h, w)
        if key in self.bufs:
            return self.bufs[key]
        t = self.torch
        bf = t.bfloat16
        B = {}
        for l, c in enumerate(LEVELS):
            hh, ww = h >> l, w >> l
            B[f"in{l}"] = self._new((n, hh, ww, IN_P if l == 0 else LEVELS[l - 1]), bf)   # conv-a input
            B[f"e{l}a"] = self._new((n, hh, ww, c), bf)
            if l < 3:
                B[f"cat{l}"] = self._new((n, hh, ww, 2 * c), bf)    # [up | encoder output]
                B[f"d{l}a"] = self._new((n, hh, ww, c), bf)
                B[f"d{l}b"] = self._new((n, hh, ww, c), bf)
            else:
                B["e3b"] = self._new((n, hh, ww, c), bf)
        B["out"] = self._new((n, h, w, OUT_P))
        G = {k: t.zeros_like(v) for k, v in B.items() if k != "out"}
        G["out"] = self._new((n, h, w, OUT_P), bf)
        self.bufs[key] = (B, G)
        return B, G

    # ---- forward / backward -------------------------------------------------
    def forward(self, x):
        """x: (n, h, w, 3) float32 CUDA tensor, h and w multiples of 8 -> (n, h, w, 3) float32."""
        n, h, w, _ = x.shape
        assert h % 8 == 0 and w % 8 == 0
        B, G = self._buffers(n, h, w)
        o, P = self.ops, self.params
        B["in0"].zero_()
        B["in0"][..., :IN_C].copy_(x)
        for l, c in enumerate(LEVELS):
            hh, ww = h >> l, w >> l
            cin = B[f"in{l}"]
            o.conv(act(cin, n, hh, ww), P[f"e{l}a"].wb, P[f"e{l}a"].b, act(B[f"e{l}a"], n, hh, ww))
            eb = act(B[f"cat{l}"], n, hh, ww, c, c) if l < 3 else act(B["e3b"], n, hh, ww)
            o.conv(act(B[f"e{l}a"], n, hh, ww), P[f"e{l}b"].wb, P[f"e{l}b"].b, eb)
            if l < 3:
                o.pool(eb, B[f"in{l + 1}"])
        prev = act(B["e3b"], n, h >> 3, w >> 3)
        for l in (2, 1, 0):
            c, hh, ww = LEVELS[l], h >> l, w >> l
            o.up(prev, P[f"u{l}"].wb, P[f"u{l}"].b, act(B[f"cat{l}"], n, hh, ww, c, 0))
            o.conv(act(B[f"cat{l}"], n, hh, ww), P[f"d{l}a"].wb, P[f"d{l}a"].b, act(B[f"d{l}a"], n, hh, ww))
            o.conv(act(B[f"d{l}a"], n, hh, ww), P[f"d{l}b"].wb, P[f"d{l}b"].b, act(B[f"d{l}b"], n, hh, ww))
            prev = act(B[f"d{l}b"], n, hh, ww)
        o.conv(prev, P["out"].wb, P["out"].b, _out_view(B["out"], n, h, w), relu=False, y32=B["out"])
        return B["out"][..., :OUT_C]

    def backward(self, gout):
        """gout: BF16 (n, h, w, OUT_P) gradient of the loss w.r.t. the output; fills p.g, p.bg."""
        n, h, w, _ = gout.shape
        B, G = self._buffers(n, h, w)
        o, P = self.ops, self.params
        for p in P.values():
            p.g.zero_()
            p.bg.zero_()
        # output convolution
        d0b = act(B["d0b"], n, h, w)
        go = act(gout, n, h, w)
        o.conv_wgrad(d0b, go, P["out"].g)
        o.bias_grad(go, P["out"].bg)
        o.conv_dgrad(go, P["out"].aux, act(G["d0b"], n, h, w), mask=d0b)
        for l in (0, 1, 2):
            c, hh, ww = LEVELS[l], h >> l, w >> l
            gdb = act(G[f"d{l}b"], n, hh, ww)
            o.conv_wgrad(act(B[f"d{l}a"], n, hh, ww), gdb, P[f"d{l}b"].g)
            o.bias_grad(gdb, P[f"d{l}b"].bg)
            o.conv_dgrad(gdb, P[f"d{l}b"].aux, act(G[f"d{l}a"], n, hh, ww), mask=act(B[f"d{l}a"], n, hh, ww))
            gda = act(G[f"d{l}a"], n, hh, ww)
            o.conv_wgrad(act(B[f"cat{l}"], n, hh, ww), gda, P[f"d{l}a"].g)
            o.bias_grad(gda, P[f"d{l}a"].bg)
            o.conv_dgrad(gda, P[f"d{l}a"].aux, act(G[f"cat{l}"], n, hh, ww), mask=act(B[f"cat{l}"], n, hh, ww))
            # transposed convolution that produced cat[:, :c]
            gup = act(G[f"cat{l}"], n, hh, ww, c, 0)
            src = act(B["e3b"] if l == 2 else B[f"d{l + 1}b"], n, hh >> 1, ww >> 1)
            o.up_wgrad(src, gup, P[f"u{l}"].g)
            o.bias_grad(gup, P[f"u{l}"].bg)
            gsrc = G["e3b"] if l == 2 else G[f"d{l + 1}b"]
            o.up_dgrad(gup, P[f"u{l}"].aux, act(gsrc, n, hh >> 1, ww >> 1), mask=src)
        # encoder, deepest first; the skip gradients already sit in cat[:, c:]
        for l in (3, 2, 1, 0):
            c, hh, ww = LEVELS[l], h >> l, w >> l
            if l == 3:
                geb, eb = act(G["e3b"], n, hh, ww), act(B["e3b"], n, hh, ww)
            else:
                geb, eb = act(G[f"cat{l}"], n, hh, ww, c, c), act(B[f"cat{l}"], n, hh, ww, c, c)
                # pooling of this level's output fed level l+1
                o.pool_bwd(eb, G[f"in{l + 1}"], geb, relu_mask=True)
            o.conv_wgrad(act(B[f"e{l}a"], n, hh, ww), geb, P[f"e{l}b"].g)
            o.bias_grad(geb, P[f"e{l}b"].bg)
            gea = act(G[f"e{l}a"], n, hh, ww)
            o.conv_dgrad(geb, P[f"e{l}b"].aux, gea, mask=act(B[f"e{l}a"], n, hh, ww))
            o.conv_wgrad(act(B[f"in{l}"], n, hh, ww), gea, P[f"e{l}a"].g)
            o.bias_grad(gea, P[f"e{l}a"].bg)
            if l > 0:
                o.conv_dgrad(gea, P[f"e{l}a"].aux, act(G[f"in{l}"], n, hh, ww))

    def loss_grad(self, x, target):
        """Forward, mean-squared error against target ((n, h, w, 3) float32) and backward:
        fills every p.g and p.bg; returns the loss (device scalar)."""
        t = self.torch
        n, h, w, _ = x.shape
        B, G = self._buffers(n, h, w)
        self.forward(x)
        loss = t.zeros(1, device=self.dev)
        cnt = n * h * w * OUT_C
        self.ops.mse(B["out"], target.contiguous(), OUT_C, 2.0 / cnt, G["out"], loss)
        self.backward(G["out"])
        return loss / cnt

    def step(self, x, target, lr=1e-3, group=None):
        """One Adam step on the MSE between forward(x) and target ((n, h, w, 3) float32).
        With torch.distributed initialised, every rank passes its own batch and the
        gradients are averaged over the ranks of `group` (data parallel, NCCL) before
        the update, so the replicas stay identical."""
        loss = self.loss_grad(x, target)
        average_gradients([t for p in self.params.values() for t in (p.g, p.bg)], group)
        self.t += 1
        for p in self.params.values():
            self.ops.adam(p.w, p.g, p.m, p.v, p.wb, lr, self.t)
            self.ops.adam(p.b, p.bg, p.bm, p.bv, p.bb, lr, self.t)
        for p in self.params.values():
            if p.kind == "conv":
                self.ops.flip3(p.wb, p.aux, p.co, p.ci)
            else:
                self.ops.transpose(p.wb, p.aux, 4 * p.co, p.ci)
        return loss

    def flops_per_sample(self, h, w):
        """Multiply-adds x 2 of one forward pass on an h x w image."""
        f = 0
        for name, p in self.params.items():
            l = int(name[1]) if name[0] in "edu" else 0
            pix = (h >> l) * (w >> l)
            if p.kind == "conv":
                f += 2 * pix * p.co * 9 * p.ci
            else:
                f += 2 * (pix // 4) * 4 * p.co * p.ci
        return f


def average_gradients(tensors, group=None):
    """All-reduce (mean) a list of gradient tensors over the ranks of `group`, as one
    flat bucket; a no-op on one process."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) < 2:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, group=group)
    flat /= dist.get_world_size(group)
    off = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[off:off + n].view_as(t))
        off += n


def _out_view(t, n, h, w):
    """ertm_nn_act describing the FP32 output's channel layout (data unused by the kernel)."""
    a = _NnAct()
    a.data, a.n, a.h, a.w, a.cstride, a.coff, a.c = t.data_ptr(), n, h, w, t.shape[-1], 0, t.shape[-1]
    return a
