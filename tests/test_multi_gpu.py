"""Several 3D shots in one launch per step (ertm_rtm_multi, GPU).

Each shot has its own context with its own grid (different nx, ny, record length
and source-pass length, the same nz); ertm_rtm_multi runs all of them with one
launch of each step kernel per time step, shots with fewer steps idling at the
end of the source pass and at the start of the receiver pass.  The per-cell
arithmetic is that of ertm_rtm_shot, so the images and the excitation state are
bit-identical to one ertm_rtm_shot per context; both stencil radii and both
boundary kinds.  Argument checks: mixed depths, 2D grids, repeated contexts,
more than ERTM_MULTI_MAX shots.
"""
import numpy as np
import pytest

from _cases import CASES, DT_MS, model, product_config

pytestmark = pytest.mark.gpu


def _shots(ertm, orc, case):
    c = CASES[case]
    nz, ny, nx = c["shape"]
    pml = c["pml"]
    grids = [(nz, ny, nx, 190, 0), (nz, ny - 5, nx - 7, 150, 90), (nz, ny - 9, nx - 3, 220, 0)]
    w = orc.ricker(25.0, DT_MS / 1000.0)
    out = []
    for q, (gz, gy, gx, nt, ns) in enumerate(grids):
        cfg = product_config(ertm, case, nt, ns)
        cfg.nx, cfg.ny = gx, gy
        vp, vs, rho = model((gz, gy, gx), seed=20 + q)
        src = (gx // 2 + q, gy // 2 - q, pml[4] + 3)
        rec = dict(rx0=pml[0], nrx=gx - pml[0] - pml[1], drx=1, ry0=pml[2],
                   nry=max(1, (gy - pml[2] - pml[3]) // 3), dry=3, rz=pml[4] + 3)
        out.append((cfg, (vp, vs, rho), ertm.Shot(*src, wavelet=w, **rec)))
    return out


def _contexts(ertm, shots):
    ctxs, data = [], []
    for cfg, m, shot in shots:
        ctx = ertm.Context(cfg)
        ctx.set_model(ertm.TRUE_MODEL, *m)
        ctx.set_model(ertm.MIGRATION_MODEL, *m)
        data.append(ctx.forward_together_using_real_model(shot))
        ctxs.append(ctx)
    return ctxs, data


@pytest.mark.parametrize("case", ["3d_r4_cpml", "3d_r6_sponge"])
def test_multi_equals_one_shot_per_context(ertm, orc, case):
    shots = _shots(ertm, orc, case)
    ctxs, data = _contexts(ertm, shots)
    ref, ref_ex = [], []
    for ctx, (cfg, m, shot), d in zip(ctxs, shots, data):
        ref.append(ctx.rtm_shot(shot, d))
        ref_ex.append(ctx.get_excitation())
    got = ertm.rtm_multi(ctxs, [s[2] for s in shots], data)
    for q, ctx in enumerate(ctxs):
        ex = ctx.get_excitation()
        for k in ("amp", "time", "evx", "evy", "evz", "etp"):
            assert np.array_equal(ex[k], ref_ex[q][k]), (q, k)
        for k in range(3):
            assert np.abs(ref[q][k]).max() > 0, (q, k)
            assert np.array_equal(got[q][k], ref[q][k]), (q, k)
    for ctx in ctxs:
        ctx.close()


def test_multi_device_arrays(ertm, orc):
    import torch
    shots = _shots(ertm, orc, "3d_r4_cpml")[:2]
    ctxs, data = _contexts(ertm, shots)
    host = ertm.rtm_multi(ctxs, [s[2] for s in shots], data)
    outs = [tuple(torch.zeros(c.cfg.shape, device="cuda") for _ in range(3)) for c in ctxs]
    ertm.rtm_multi(ctxs, [s[2] for s in shots], [torch.from_numpy(d).cuda() for d in data], outs)
    for h, o in zip(host, outs):
        for k in range(3):
            assert np.array_equal(o[k].cpu().numpy(), h[k])
    for ctx in ctxs:
        ctx.close()


def test_multi_argument_checks(ertm, orc):
    shots = _shots(ertm, orc, "3d_r4_cpml")
    ctxs, data = _contexts(ertm, shots[:2])
    sh = [s[2] for s in shots[:2]]
    with pytest.raises(ertm.ErtmError):
        ertm.rtm_multi([ctxs[0], ctxs[0]], [sh[0], sh[0]], [data[0], data[0]])
    cfg, m, shot = shots[0]
    deeper = ertm.Context(ertm.Config(**{**cfg.__dict__, "nz": cfg.nz + 2}))
    vp, vs, rho = model(deeper.cfg.shape, seed=3)
    deeper.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
    with pytest.raises(ertm.ErtmError):
        ertm.rtm_multi([ctxs[0], deeper], [sh[0], sh[0]], [data[0], data[0]])
    flat = ertm.Context(product_config(ertm, "2d_r4_cpml", 50))
    vp, vs, rho = model(flat.cfg.shape, seed=4)
    flat.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
    fshot = ertm.Shot(40, 0, 15, wavelet=orc.ricker(25.0, DT_MS / 1000.0), rx0=12, nrx=60, drx=1, rz=15)
    with pytest.raises(ertm.ErtmError):
        ertm.rtm_multi([flat], [fshot], [np.zeros((3, 50, 60), np.float32)])
    with pytest.raises(ValueError):
        ertm.rtm_multi(ctxs * 6, sh * 6, data * 6)
    for ctx in ctxs + [deeper, flat]:
        ctx.close()
