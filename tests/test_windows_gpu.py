"""Batched RTM over aperture windows of a shared model (ertm_rtm_windows, GPU):
the stacked images equal the sum of one-window-per-context migrations, with one
and three 3D shots per launch and the z-chunk autotuner on, and do not depend on
the group size; two windows against the FP64 oracle."""
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
    outs = []
    for lanes in (1, 3):
        out = ertm.rtm_windows(base, *mig, wins, eshots, data, lanes=lanes)
        outs.append(out)
        for k in range(3):
            r = ref[k]
            ok = np.isfinite(r)
            scale = np.abs(r[ok]).max()
            assert scale > 0
            err = np.abs(out[k][ok] - r[ok]).max() / scale
            assert err < 1e-5, (lanes, k, err)
    # the shots are stacked in one order whatever the group size
    for k in range(3):
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_windows_match_the_oracle(ertm, orc):
    """The batched path against the FP64 oracle: two non-overlapping 2D windows, the
    oracle's modelling, source and receiver passes on each window's cropped and
    padded model, its images placed into the stack; compared on the cells whose
    excitation is tie-free (as the parity tests do), relative L2 1e-4."""
    shape = (40, 1, 160)
    nz, ny, nx = shape
    true = shared_model(shape, seed=5)
    wins = [ertm.Window(6, 0, 60, 1, 220), ertm.Window(90, 0, 56, 1, 200)]
    w = orc.ricker(25.0, DT_MS / 1000.0)
    shots, data = [], []
    ref = [np.zeros(shape) for _ in range(3)]
    clear = np.zeros(shape, bool)
    for win in wins:
        m = [crop_pad(a, win.x0, 0, win.wx, 1, PML, True) for a in true]
        wnz, _, wnx = m[0].shape
        s = dict(sx=win.x0 + win.wx // 2, sy=0, sz=2, rx0=win.x0, nrx=(win.wx + 1) // 2, drx=2,
                 ry0=0, nry=1, dry=2, rz=2)
        g = orc.make_grid(wnx, 1, wnz, 10.0, 10.0, 10.0, DT_MS, R=4, boundary=orc.CPML,
                          pml=(PML, PML, 0, 0, PML, PML), pml_vmax=float(m[0].max()))
        osh = orc.make_shot(s["sx"] - win.x0 + PML, 0, s["sz"] + PML, w, rx0=s["rx0"] - win.x0 + PML,
                            nrx=s["nrx"], drx=2, rz=s["rz"] + PML)
        d = orc.run_pass(g, *m, osh, orc.MODEL, win.nt)["data"]
        nsrc = 2 * win.nt // 3
        ex = orc.run_pass(g, *m, osh, orc.SOURCE, nsrc)["ex"]
        r = orc.run_pass(g, *m, osh, orc.RECEIVER, win.nt, data=d, ex=ex)
        ok = (ex.amp2 - ex.second2 > 2e-4 * ex.amp2) & (ex.amp2 > 1e-4 * np.percentile(ex.amp2, 99))
        for k, name in enumerate(("pp", "ps")):
            ref[k][:, :, win.x0:win.x0 + win.wx] = r[name][PML:PML + nz, :, PML:PML + win.wx]
        clear[:, :, win.x0:win.x0 + win.wx] = ok[PML:PML + nz, :, PML:PML + win.wx]
        shots.append(ertm.Shot(s["sx"], 0, s["sz"], wavelet=w, rx0=s["rx0"], nrx=s["nrx"], drx=2, rz=s["rz"]))
        data.append(d)
    base = config(ertm, nx, ny, nz, 1, True)
    out = ertm.rtm_windows(base, *true, wins, shots, data, lanes=2)
    assert clear.sum() > 1000
    for k in range(2):
        got, want = out[k][clear], ref[k][clear]
        err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
        assert err <= 1e-4, (k, err)
