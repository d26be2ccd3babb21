"""Batched RTM over aperture windows of a shared model (ertm_rtm_windows, GPU):
the stacked images equal the sum of one-window-per-context migrations, with
several lanes in flight and the z-chunk autotuner on."""
import numpy as np
import pytest

from _windows_case import (DT_MS, PML, config, crop_pad, shared_model, to_window_shot,
                           windows)

pytestmark = pytest.mark.gpu


def _reference(ertm, orc, true, mig, wins, shots, two_d, shape):
    nz, ny, nx = shape
    w = orc.ricker(25.0, DT_MS / 1000.0)
    stack = [np.zeros(shape, np.float64) for _ in range(3)]
    data = []
    for win, s in zip(wins, shots):
        mt = [crop_pad(a, win.x0, win.y0, win.wx, win.wy, PML, two_d) for a in true]
        mm = [crop_pad(a, win.x0, win.y0, win.wx, win.wy, PML, two_d) for a in mig]
        wnz, wny, wnx = mt[0].shape
        ctx = ertm.Context(config(ertm, wnx, wny, wnz, win.nt, two_d))
        ctx.set_model(ertm.TRUE_MODEL, *mt)
        ctx.set_model(ertm.MIGRATION_MODEL, *mm)
        sh = to_window_shot(ertm, s, win, two_d, w)
        d = ctx.forward_together_using_real_model(sh)
        data.append(d)
        imgs = ctx.rtm_shot(sh, d)
        ys = slice(0, 1) if two_d else slice(PML, PML + win.wy)
        for k in range(3):
            part = imgs[k][PML:PML + nz, ys, PML:PML + win.wx]
            stack[k][:, win.y0:win.y0 + (1 if two_d else win.wy), win.x0:win.x0 + win.wx] += part
        ctx.close()
    return stack, data, w


@pytest.mark.parametrize("two_d", [False, True])
def test_windows_equal_per_window_contexts(ertm, orc, two_d):
    shape = (40, 1, 160) if two_d else (36, 60, 72)
    nz, ny, nx = shape
    true = shared_model(shape)
    mig = tuple(np.ascontiguousarray(a) for a in true)   # same model: strong images
    wins, shots = windows(ertm, shape, 5, seed=7, two_d=two_d, wmin=24, wmax=48 if not two_d else 100,
                          ntmin=150, ntmax=230)
    ref, data, w = _reference(ertm, orc, true, mig, wins, shots, two_d, shape)
    eshots = [ertm.Shot(s["sx"], s["sy"], s["sz"], wavelet=w, rx0=s["rx0"], nrx=s["nrx"], drx=s["drx"],
                        ry0=s["ry0"], nry=s["nry"], dry=s["dry"], rz=s["rz"]) for s in shots]
    base = config(ertm, nx, ny, nz, 1, two_d, autotune=1)
    for lanes in (1, 3):
        out = ertm.rtm_windows(base, *mig, wins, eshots, data, lanes=lanes)
        for k in range(3):
            r = ref[k]
            ok = np.isfinite(r)
            scale = np.abs(r[ok]).max()
            assert scale > 0
            err = np.abs(out[k][ok] - r[ok]).max() / scale
            assert err < 1e-5, (lanes, k, err)
