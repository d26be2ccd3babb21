"""Learned-preconditioned LSRTM: training pairs from the method itself, U-Net
training on them, and CG with the network as its preconditioner.

For each seeded layered-and-faulted 2D model the migration model is the
Gaussian-smoothed true model, the reflectivity is the relative perturbation
(true / smooth - 1) of (vp, vs, rho), and the observed data are its Born data
(`Context.born_forward`).  A training pair is (first gradient F^T d, reflectivity
after `cg_iters` CG iterations); both are normalised by their RMS, so the
network learns the shape of the CG result from the shape of the gradient.  In
CG the preconditioner applies the network to the current gradient; plain CG
stays the fallback (lsrtm.cgls accepts a preconditioned step only if the
Born-modelled data misfit falls).
"""
from __future__ import annotations

import json
import time
from dataclasses import dataclass, field

import numpy as np

from . import (BOUNDARY_SPONGE_CUBIC, MIGRATION_MODEL, Config, Context, Shot)
from . import lsrtm as _lsrtm
from . import synthetic as _syn


@dataclass
class Case:
    ctx: Context
    shots: list
    data: list
    true: tuple          # relative perturbations (r_vp, r_vs, r_rho), (nz, 1, nx)
    shape: tuple


@dataclass
class Geometry:
    nzi: int = 64        # interior cells
    nxi: int = 128
    h: float = 10.0
    pml: int = 20
    nt: int = 500
    dt_ms: float = 1.0
    nshots: int = 6
    f0: float = 15.0
    sigma: float = 4.0   # smoothing of the migration model, cells
    visco: tuple | None = None


def make_case(seed: int, g: Geometry, device: int = 0, checkpoint_every: int = 100) -> Case:
    vp, vs, rho = _syn.faulted_2d(seed, g.nzi, g.nxi, g.h, vmax=3500.0)
    pads = (g.pml, g.pml, 0, 0, g.pml, g.pml)
    vp, vs, rho = (_syn.pad_edges(a, pads) for a in (vp, vs, rho))
    svp, svs, srho = (_syn.gaussian_smooth(a, g.sigma) for a in (vp, vs, rho))
    true = tuple((a / b - 1.0).astype(np.float32) for a, b in ((vp, svp), (vs, svs), (rho, srho)))
    nz, _, nx = vp.shape
    v = dict(zip(("visco_nmech", "visco_qp", "visco_qs", "visco_f0"), g.visco)) if g.visco else {}
    cfg = Config(nx=nx, ny=1, nz=nz, dx=g.h, dy=g.h, dz=g.h, dt_ms=g.dt_ms, nt=g.nt, order=8,
                 boundary=BOUNDARY_SPONGE_CUBIC, pml=pads, sponge_coef=150.0,
                 checkpoint_every=checkpoint_every, device=device, **v)
    ctx = Context(cfg)
    ctx.set_model(MIGRATION_MODEL, svp, svs, srho)
    w = _syn.ricker(g.f0, g.dt_ms / 1000.0)
    xs = np.linspace(g.pml + 4, nx - g.pml - 5, g.nshots).round().astype(int)
    rz = g.pml + 2
    shots = [Shot(int(x), 0, rz, wavelet=w, rx0=g.pml, nrx=nx - 2 * g.pml, drx=1, rz=rz) for x in xs]
    data = list(ctx.born_forward_shots(shots, *true))   # every shot in one batched call
    return Case(ctx, shots, data, true, vp.shape)


def _rms(a) -> float:
    return float(np.sqrt(np.mean(np.concatenate([x.ravel() for x in a]).astype(np.float64) ** 2))) or 1.0


def to_image(m, pad_to: int = 8) -> np.ndarray:
    """(3 volumes (nz, 1, nx)) -> (nz', nx', 3) float32, zero-padded to multiples of pad_to."""
    nz, _, nx = m[0].shape
    pz, px = -nz % pad_to, -nx % pad_to
    img = np.zeros((nz + pz, nx + px, 3), np.float32)
    for c in range(3):
        img[:nz, :nx, c] = m[c][:, 0, :]
    return img


def from_image(img, shape) -> tuple:
    nz, _, nx = shape
    return tuple(np.ascontiguousarray(img[:nz, :nx, c][:, None, :], dtype=np.float32) for c in range(3))


def training_pair(case: Case, cg_iters: int = 10):
    g = _lsrtm.adjoint_all(case.ctx, case.shots, case.data)
    res = _lsrtm.cgls(case.ctx, case.shots, case.data, niter=cg_iters)
    return to_image(g) / _rms(g), to_image(res.m) / _rms(res.m)


@dataclass
class TrainLog:
    loss: list = field(default_factory=list)
    seconds: float = 0.0
    steps: int = 0


def train(net, pairs, steps: int, batch: int, patch=(64, 128), lr: float = 1e-3, seed: int = 0,
          log_every: int = 50, log: str | None = None) -> TrainLog:
    """Adam on random patches of the (input, target) image pairs (each (H, W, 3));
    `log` (optional) is a JSON-lines file that gets the loss every `log_every` steps."""
    import torch
    rng = np.random.default_rng(seed)
    dev = net.dev
    X = [torch.from_numpy(x).to(dev) for x, _ in pairs]
    Y = [torch.from_numpy(y).to(dev) for _, y in pairs]
    ph, pw = patch
    tl = TrainLog()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    xb = torch.zeros((batch, ph, pw, 3), device=dev)
    yb = torch.zeros((batch, ph, pw, 3), device=dev)
    for it in range(steps):
        for b in range(batch):
            k = int(rng.integers(len(X)))
            H, W = X[k].shape[:2]
            i0 = int(rng.integers(0, H - ph + 1)) if H > ph else 0
            j0 = int(rng.integers(0, W - pw + 1)) if W > pw else 0
            xb[b].zero_()
            yb[b].zero_()
            hh, ww = min(ph, H), min(pw, W)
            xb[b, :hh, :ww] = X[k][i0:i0 + hh, j0:j0 + ww]
            yb[b, :hh, :ww] = Y[k][i0:i0 + hh, j0:j0 + ww]
        loss = net.step(xb, yb, lr=lr)
        if it % log_every == 0 or it == steps - 1:
            tl.loss.append((it, float(loss.item())))
            if log:
                with open(log, "a") as f:
                    f.write(json.dumps({"event": "unet_step", "step": it, "loss": tl.loss[-1][1]}) + "\n")
    torch.cuda.synchronize(dev)
    tl.seconds = time.perf_counter() - t0
    tl.steps = steps
    return tl


def preconditioner(net, shape):
    """CG preconditioner: the network applied to the RMS-normalised gradient."""
    import torch

    def P(s):
        img = to_image(s)
        x = torch.from_numpy(img[None] / _rms(s)).to(net.dev)
        y = net.forward(x).float().cpu().numpy()[0]
        return from_image(y, shape)

    return P


def iters_to(misfit: list, target: float):
    for i, m in enumerate(misfit):
        if m <= target:
            return i + 1
    return None


def _model_err(m, ref) -> float:
    num = sum(float(np.sum((a.astype(np.float64) - b) ** 2)) for a, b in zip(m, ref))
    den = sum(float(np.sum(b.astype(np.float64) ** 2)) for b in ref)
    return float(np.sqrt(num / max(den, 1e-30)))


def compare(case: Case, net, niter: int, target: float):
    """Plain vs learned-preconditioned CG on one case: misfit curves; iterations and
    wall time to reach `target` and to reach plain CG's final (niter-th) misfit;
    reflectivity errors against the true perturbation."""
    t0 = time.perf_counter()
    plain = _lsrtm.cgls(case.ctx, case.shots, case.data, niter=niter)
    tp = time.perf_counter() - t0
    t0 = time.perf_counter()
    learned = _lsrtm.cgls(case.ctx, case.shots, case.data, niter=niter,
                          precond=preconditioner(net, case.shape))
    tl = time.perf_counter() - t0
    ip, il = iters_to(plain.misfit, target), iters_to(learned.misfit, target)
    per_p, per_l = tp / max(1, len(plain.misfit)), tl / max(1, len(learned.misfit))
    pfin = plain.misfit[-1]
    il_fin = iters_to(learned.misfit, pfin)
    return {"plain_misfit": plain.misfit, "learned_misfit": learned.misfit,
            "accepted": learned.accepted, "plain_iters": ip, "learned_iters": il,
            "plain_seconds": tp, "learned_seconds": tl,
            "plain_time_to_target": ip * per_p if ip else None,
            "learned_time_to_target": il * per_l if il else None,
            "learned_iters_to_plain_final": il_fin,
            "learned_time_to_plain_final": il_fin * per_l if il_fin else None,
            "time_ratio_to_plain_final": (il_fin * per_l) / tp if il_fin else None,
            "plain_model_err": _model_err(plain.m, case.true),
            "learned_model_err": _model_err(learned.m, case.true),
            "model_rel_diff": _model_err(learned.m, plain.m)}
