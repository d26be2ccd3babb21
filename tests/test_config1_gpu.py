"""The reference's CPU-runnable case at full size (2D, 600 x 300 interior at 5 m
plus a 40-cell C-PML, three layers and a Gaussian lens, 15 Hz Ricker, nt 3000,
600 receivers): observed data and the RTM images of the CUDA path against the
FP64 oracle (GPU).  Tolerances as in test_parity_gpu.py."""
import importlib

import numpy as np
import pytest

from _cases import rel

pytestmark = pytest.mark.gpu

TIE, FLOOR = 2e-4, 1e-4


def test_config1_modelling_and_rtm_against_the_oracle(ertm, orc):
    synth = importlib.import_module("2d_and_3d_elastic_reverse_time_migration_b200.synthetic")
    wl = synth.layered_2d()
    nz, ny, nx = wl.shape
    nt, nsrc = wl.nt, 2 * wl.nt // 3
    w = synth.ricker(wl.freq, wl.dt_ms / 1000.0)
    pml = (wl.pml, wl.pml, 0, 0, wl.pml, wl.pml)
    g = orc.make_grid(nx, ny, nz, wl.dx, wl.dy, wl.dz, wl.dt_ms, R=4, boundary=orc.CPML, pml=pml,
                      pml_vmax=float(wl.vp.max()))
    gs = orc.make_grid(nx, ny, nz, wl.dx, wl.dy, wl.dz, wl.dt_ms, R=4, boundary=orc.CPML, pml=pml,
                       pml_vmax=float(wl.svp.max()))
    oshot = orc.make_shot(*wl.src, w, **wl.rec)
    ctx = ertm.Context(ertm.Config(nx=nx, ny=ny, nz=nz, dx=wl.dx, dy=wl.dy, dz=wl.dz, dt_ms=wl.dt_ms,
                                   nt=nt, order=8, boundary=ertm.BOUNDARY_CPML, pml=pml))
    ctx.set_model(ertm.TRUE_MODEL, wl.vp, wl.vs, wl.rho)
    ctx.set_model(ertm.MIGRATION_MODEL, wl.svp, wl.svs, wl.srho)
    pshot = ertm.Shot(*wl.src, wavelet=w, **wl.rec)

    ref = orc.run_pass(g, wl.vp, wl.vs, wl.rho, oshot, orc.MODEL, nt, bits=64)["data"]
    r32 = orc.run_pass(g, wl.vp, wl.vs, wl.rho, oshot, orc.MODEL, nt, bits=32)["data"]
    data = ctx.forward_together_using_real_model(pshot)
    for q in (0, 2):
        e, e32 = rel(data[q], ref[q]), rel(r32[q], ref[q])
        assert e <= max(1e-5, 3 * e32), (q, e, e32)

    src = orc.run_pass(gs, wl.svp, wl.svs, wl.srho, oshot, orc.SOURCE, nsrc, bits=64)
    ex = src["ex"]
    rec = orc.run_pass(gs, wl.svp, wl.svs, wl.srho, oshot, orc.RECEIVER, nt, data=ref, ex=ex, bits=64)
    ctx.forward_together_using_smoothed_model(pshot)
    gx = ctx.get_excitation()
    clear = (ex.amp2 - ex.second2 > TIE * ex.amp2) & (ex.amp2 > FLOOR * np.percentile(ex.amp2, 99))
    assert clear.mean() > 0.5
    assert not ((gx["time"] != ex.time) & clear).any()
    pp, ps, tp = ctx.backward_together_using_smoothed_model(pshot, ref)
    for name, a, b in (("pp", pp, rec["pp"]), ("ps", ps, rec["ps"])):
        assert np.isfinite(a[clear]).all(), name
        e = rel(a[clear], b[clear])
        assert e <= 1e-4, (name, e)
