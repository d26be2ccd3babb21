"""Analytic and structural properties of the CPU oracle (no GPU)."""
import numpy as np
import pytest


def _homog(orc, nx=60, ny=1, nz=56, boundary=0, R=4, pml=10):
    vp = np.full((nz, ny, nx), 3000.0, np.float32)
    vs = (vp / np.sqrt(3)).astype(np.float32)
    rho = (310 * vp ** 0.25).astype(np.float32)
    pm = (pml, pml, 0 if ny == 1 else pml, 0 if ny == 1 else pml, pml, pml)
    g = orc.make_grid(nx, ny, nz, 10.0, 10.0, 10.0, 1.0, R=R, boundary=boundary, pml=pm,
                      pml_vmax=3000.0, sponge_coef=300.0)
    return g, vp, vs, rho


def test_explosive_source_mirror_symmetry_2d(orc):
    # nx odd and the source on the centre column: the C-PML layout is mirror symmetric
    g, vp, vs, rho = _homog(orc, nx=61)
    w = orc.ricker(15.0, 1e-3)
    s = orc.make_shot(30, 0, 28, w)
    f = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 60, want_fields=True)["fields"]
    txx, tzz, vx = f["txx"][:, 0, :], f["tzz"][:, 0, :], f["vx"][:, 0, :]
    # normal stresses are even about x = sx; vx (at i-1/2) is odd: vx[sx+d] = -vx[sx-d+1]
    for d in range(1, 20):
        assert np.allclose(txx[:, 30 + d], txx[:, 30 - d], rtol=1e-9, atol=1e-12 * abs(txx).max())
        assert np.allclose(vx[:, 30 + d], -vx[:, 30 - d + 1], rtol=1e-9, atol=1e-12 * abs(vx).max())
    assert abs(tzz).max() > 0


def test_linearity_in_source(orc):
    g, vp, vs, rho = _homog(orc, nx=40, nz=40)
    w = orc.ricker(15.0, 1e-3)
    s1 = orc.make_shot(20, 0, 20, w, rx0=5, nrx=30, drx=1, rz=8)
    s2 = orc.make_shot(20, 0, 20, 2 * w, rx0=5, nrx=30, drx=1, rz=8)
    d1 = orc.run_pass(g, vp, vs, rho, s1, orc.MODEL, 80)["data"]
    d2 = orc.run_pass(g, vp, vs, rho, s2, orc.MODEL, 80)["data"]
    assert np.allclose(d2, 2 * d1, rtol=1e-6, atol=1e-7 * abs(d1).max())


@pytest.mark.parametrize("boundary", [0, 1])
def test_fp32_build_tracks_fp64(orc, boundary):
    g, vp, vs, rho = _homog(orc, nx=48, ny=40, nz=44, boundary=boundary, pml=8)
    w = orc.ricker(15.0, 1e-3)
    s = orc.make_shot(24, 20, 22, w, rx0=8, nrx=32, drx=1, ry0=20, nry=1, rz=10)
    a = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 150, want_fields=True, bits=64)
    b = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 150, want_fields=True, bits=32)
    for name in ("vx", "vz", "txx", "txy"):
        x, y = a["fields"][name], b["fields"][name]
        assert np.linalg.norm(x - y) / np.linalg.norm(x) < 1e-4, name


def test_cpml_absorbs(orc):
    """Energy left after the wave has crossed the C-PML is far below the peak."""
    g, vp, vs, rho = _homog(orc, nx=80, nz=80, pml=20)
    w = orc.ricker(15.0, 1e-3)
    s = orc.make_shot(40, 0, 40, w)
    e_peak = None
    for n in (60, 500):
        f = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, n, want_fields=True)["fields"]
        e = float(np.sum(f["vx"] ** 2 + f["vz"] ** 2))
        e_peak = e if e_peak is None else e_peak
    assert e < 1e-3 * e_peak


def test_divcurl_explosive_is_mostly_p(orc):
    g, vp, vs, rho = _homog(orc, nx=64, nz=64)
    w = orc.ricker(10.0, 1e-3)
    s = orc.make_shot(32, 0, 32, w)
    f = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 120, want_fields=True)["fields"]
    p, _, sy, _ = orc.divcurl(g, vp, vs, f["vx"], f["vy"], f["vz"])
    assert np.abs(sy).max() < 0.1 * np.abs(p).max()


def test_source_receiver_pass_images(orc):
    """Excitation capture then imaging: times lie in [0, nsrc), images finite."""
    g, vp, vs, rho = _homog(orc, nx=48, nz=48, pml=8)
    w = orc.ricker(15.0, 1e-3)
    s = orc.make_shot(24, 0, 12, w, rx0=8, nrx=32, drx=1, rz=12)
    d = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 120)["data"]
    src = orc.run_pass(g, vp, vs, rho, s, orc.SOURCE, 80)
    ex = src["ex"]
    assert ex.time.min() >= 0 and ex.time.max() < 80
    assert (ex.second2 <= ex.amp2).all()
    rec = orc.run_pass(g, vp, vs, rho, s, orc.RECEIVER, 120, data=d, ex=ex)
    for k in ("pp", "ps", "tp"):
        assert np.isfinite(rec[k]).all()
    assert np.abs(rec["pp"]).max() > 0


@pytest.mark.parametrize("boundary", [0, 1])
def test_explosive_source_xy_transpose_symmetry_3d(orc, boundary):
    """The 3D y terms (restated from the 2D x terms; the reference's 3D kernels are
    absent) treat y exactly like x: with a cube-symmetric setup, swapping x and y
    maps tp, txx<->tyy, txy onto themselves and vx onto vy (vx at i-1/2 and vy at
    j-1/2 swap places)."""
    n = 33
    g, vp, vs, rho = _homog(orc, nx=n, ny=n, nz=30, boundary=boundary, pml=8)
    w = orc.ricker(18.0, 1e-3)
    s = orc.make_shot(16, 16, 14, w)
    f = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 45, want_fields=True)["fields"]
    T = lambda a: a.transpose(0, 2, 1)
    scale = lambda a: 1e-10 * abs(a).max()
    assert np.allclose(f["txx"], T(f["tyy"]), rtol=1e-9, atol=scale(f["txx"]))
    assert np.allclose(f["tzz"], T(f["tzz"]), rtol=1e-9, atol=scale(f["tzz"]))
    assert np.allclose(f["txy"], T(f["txy"]), rtol=1e-9, atol=scale(f["txy"]))
    assert np.allclose(f["txz"], T(f["tyz"]), rtol=1e-9, atol=scale(f["txz"]))
    assert np.allclose(f["vx"], T(f["vy"]), rtol=1e-9, atol=scale(f["vx"]))
    assert abs(f["vx"]).max() > 0 and abs(f["txy"]).max() > 0


def test_p_travel_time_3d(orc):
    """Known answer for the 3D scheme: between receivers 12 and 24 cells from an
    explosive source (on the x axis), the P wave's travel time is 12 cells / vp —
    measured as the lag of the cross-correlation of the two vx traces."""
    n = 61
    g, vp, vs, rho = _homog(orc, nx=n, ny=n, nz=n, boundary=0, pml=10)
    dt = 1e-3
    w = orc.ricker(12.0, dt)
    c = 30
    s = orc.make_shot(c, c, c, w, rx0=c + 12, nrx=2, drx=12, ry0=c, nry=1, dry=1, rz=c)
    data = orc.run_pass(g, vp, vs, rho, s, orc.MODEL, 200)["data"]
    a, b = data[0, :, 0].astype(np.float64), data[0, :, 1].astype(np.float64)
    xc = np.correlate(b, a, mode="full")
    lag = int(np.argmax(xc)) - (len(a) - 1)
    expect = 12 * 10.0 / 3000.0 / dt                          # 40 steps
    assert abs(lag - expect) <= 1, (lag, expect)
