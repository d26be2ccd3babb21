"""Parity at the 3D workload's own grid (GPU): 480 x 480 x 380 cells.

The bench times the 400 x 400 x 300 interior with its 40-cell C-PML
(480 x 480 x 380 = 87.55 M cells, R = 4, dt 0.8 ms) on the seeded layered model
with the ellipsoid.  This test runs the CUDA path on that exact grid and model
and compares it with the FP64 oracle on the host cores: 120 modelling steps
(all nine wavefields and the surface traces) and a 120-step source pass
(excitation time and amplitude).  At this size the cell offsets are near their
32-bit range, every column has 12 z chunks and 45 % of the cells lie in C-PML
slabs.  The source sits 8 cells inside the x-, y- and z-minimum slabs, so in
120 steps the wavefield crosses three slab faces and the slab corners; a
25 Hz Ricker (107 samples) ends inside the pass, so every cell near the source
sees its whole first arrival.  The reference's 3D driver loop is
3D_elastic_RTM/3D_forward_or_back_together.cu:9-290.

Tolerances: flat relative L2 <= 1e-5 for wavefields and traces; excitation
time bit-exact on tie-free cells; excitation amplitude relative L2 <= 1e-4.
The oracle needs about 35 GB of host memory and a few minutes of host time.
"""
import numpy as np
import pytest

from _cases import rel

pytestmark = pytest.mark.gpu

NSTEPS = 120
FREQ = 25.0
TIE, FLOOR = 2e-4, 1e-4
FIELDS3 = ("vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz")


def _host_gb():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


@pytest.fixture(scope="module")
def case(ertm, orc, synth):
    if _host_gb() < 48:
        pytest.skip(f"needs ~48 GB of free host memory for the FP64 oracle, {_host_gb():.0f} GB free")
    wl = synth.layered_3d(smooth_sigma=0)      # the bench's seeded model, unsmoothed
    nz, ny, nx = wl.shape
    assert (nz, ny, nx) == (380, 480, 480)
    p = wl.pml
    src = (p + 8, p + 8, p + 8)
    w = orc.ricker(FREQ, wl.dt_ms / 1000.0)
    g = orc.make_grid(nx, ny, nz, wl.dx, wl.dy, wl.dz, wl.dt_ms, R=4, boundary=orc.CPML,
                      pml=(p,) * 6, pml_r=1e-3, pml_f0=10.0, pml_vmax=float(wl.vp.max()))
    cfg = ertm.Config(nx=nx, ny=ny, nz=nz, dx=wl.dx, dy=wl.dy, dz=wl.dz, dt_ms=wl.dt_ms, nt=NSTEPS,
                      src_steps=NSTEPS, order=8, boundary=ertm.BOUNDARY_CPML, pml=(p,) * 6,
                      pml_r=1e-3, pml_f0=10.0)
    return dict(wl=wl, src=src, w=w, g=g, cfg=cfg, oshot=orc.make_shot(*src, w, **wl.rec),
                pshot=ertm.Shot(*src, wavelet=w, **wl.rec))


def test_config2_grid_wavefields_and_traces(ertm, orc, case):
    wl = case["wl"]
    ref = orc.run_pass(case["g"], wl.vp, wl.vs, wl.rho, case["oshot"], orc.MODEL, NSTEPS,
                       want_fields=True, bits=64)
    with ertm.Context(case["cfg"]) as ctx:
        ctx.set_model(ertm.TRUE_MODEL, wl.vp, wl.vs, wl.rho)
        data = ctx.forward_together_using_real_model(case["pshot"])
        report = {}
        for name in FIELDS3:
            report[name] = rel(ctx.get_wavefield(name), ref["fields"][name])
    for q in range(3):
        report[f"trace{q}"] = rel(data[q], ref["data"][q])
    print("480x480x380, 120 steps, relative L2 against FP64:", report)
    bad = {k: v for k, v in report.items() if not v <= 1e-5}
    assert not bad, bad


def test_config2_grid_excitation(ertm, orc, case):
    wl = case["wl"]
    ex = orc.run_pass(case["g"], wl.vp, wl.vs, wl.rho, case["oshot"], orc.SOURCE, NSTEPS,
                      bits=64)["ex"]
    with ertm.Context(case["cfg"]) as ctx:
        ctx.set_model(ertm.MIGRATION_MODEL, wl.vp, wl.vs, wl.rho)
        ctx.forward_together_using_smoothed_model(case["pshot"])
        gx = ctx.get_excitation()
    excited = ex.amp2 > FLOOR * np.percentile(ex.amp2[ex.amp2 > 0], 99)
    clear = (ex.amp2 - ex.second2 > TIE * ex.amp2) & excited
    assert clear.sum() > 10000, int(clear.sum())
    mism = (gx["time"] != ex.time) & clear
    assert not mism.any(), f"{int(mism.sum())} of {int(clear.sum())} tie-free cells differ in time"
    amp_ref = np.sqrt(ex.amp2.astype(np.float64))
    e = rel(gx["amp"][clear], amp_ref[clear])
    print(f"tie-free excited cells {int(clear.sum())}, amplitude relative L2 {e:.2e}")
    assert e <= 1e-4
