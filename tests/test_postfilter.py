"""Image and gradient post-filters against numpy restatements of the reference's
cpu_laplace / suhilbt (zzzzz:1018-1066, 1110-1147) and of its GPU smoothing and
taper kernels (2D_elastic_RTM/viscoelastic_equation.cu:2528-2604, 2881-2926)."""
import numpy as np
import pytest


def _laplace_ref(r, vp, h):
    """numpy restatement of cpu_laplace (2D; every column's top/bottom edge copied)"""
    nz, _, nx = r.shape
    a = r[:, 0, :].astype(np.float64)
    t = -a.copy()
    t[1:-1, 1:-1] = -((a[1:-1, 2:] + a[1:-1, :-2] - 2 * a[1:-1, 1:-1]) / h[0] ** 2 +
                      (a[2:, 1:-1] + a[:-2, 1:-1] - 2 * a[1:-1, 1:-1]) / h[2] ** 2)
    t[:, 0], t[:, -1] = t[:, 1], t[:, -2]
    t[0, :], t[-1, :] = t[1, :], t[-2, :]
    return (vp[:, 0, :].astype(np.float64) ** 2 * t / 4)[:, None, :]


def test_laplace_filter(ertm):
    rng = np.random.default_rng(4)
    r = rng.standard_normal((30, 1, 41)).astype(np.float32)
    vp = (2000 + 500 * rng.random((30, 1, 41))).astype(np.float32)
    out = ertm.laplace_filter(r, vp, (5.0, 5.0, 4.0))
    ref = _laplace_ref(r, vp, (5.0, 5.0, 4.0))
    assert np.allclose(out, ref, rtol=1e-4, atol=1e-3 * np.abs(ref).max())



def test_laplace_filter_3d(ertm):
    rng = np.random.default_rng(10)
    r = rng.standard_normal((12, 9, 14)).astype(np.float64)
    vp = (2000 + 500 * rng.random(r.shape)).astype(np.float32)
    h = (5.0, 6.0, 4.0)
    t = -r.copy()
    c = r[1:-1, 1:-1, 1:-1]
    t[1:-1, 1:-1, 1:-1] = -((r[1:-1, 1:-1, 2:] + r[1:-1, 1:-1, :-2] - 2 * c) / h[0] ** 2 +
                            (r[1:-1, 2:, 1:-1] + r[1:-1, :-2, 1:-1] - 2 * c) / h[1] ** 2 +
                            (r[2:, 1:-1, 1:-1] + r[:-2, 1:-1, 1:-1] - 2 * c) / h[2] ** 2)
    t[:, :, 0], t[:, :, -1] = t[:, :, 1], t[:, :, -2]
    t[:, 0, :], t[:, -1, :] = t[:, 1, :], t[:, -2, :]
    t[0], t[-1] = t[1], t[-2]
    ref = vp.astype(np.float64) ** 2 * t / 4
    out = ertm.laplace_filter(r.astype(np.float32), vp, h)
    assert np.allclose(out, ref, rtol=1e-4, atol=1e-4 * np.abs(ref).max())
    with pytest.raises(ertm.ErtmError):
        ertm.laplace_filter(np.zeros((2, 1, 5), np.float32), np.ones((2, 1, 5), np.float32), h)

def test_hilbert_transform_along_depth(ertm):
    nz = 64
    z = np.arange(nz)
    col = np.cos(2 * np.pi * 5 * z / nz).astype(np.float32)
    img = np.repeat(col[:, None, None], 3, axis=2)
    out = ertm.hilbert_z(img)
    # the Hilbert transform of cos is sin (sign convention of the reference: -i for
    # the first half of the spectrum)
    assert np.allclose(out[:, 0, 0], np.sin(2 * np.pi * 5 * z / nz), atol=1e-5)
    r = np.random.default_rng(5).standard_normal((37, 2, 3)).astype(np.float32)
    X = np.fft.fft(r.astype(np.float64), axis=0)
    H = np.where(np.arange(37)[:, None, None] < 37 // 2, -1j, 1j)
    ref = np.real(np.fft.ifft(X * H, axis=0))
    assert np.allclose(ertm.hilbert_z(r), ref, atol=1e-5)



def _bell2d_ref(g, r):
    """cuda_bell_smooth_2d restated directly: the full truncated 2D window, one sum."""
    nz, nx = g.shape
    out = np.zeros_like(g, dtype=np.float64)
    for iz in range(nz):
        for ix in range(nx):
            z0, z1 = max(0, iz - r), min(nz, iz + r + 1)
            x0, x1 = max(0, ix - r), min(nx, ix + r + 1)
            dz = np.arange(z0, z1) - iz
            dx = np.arange(x0, x1) - ix
            w = np.exp(-(dz[:, None] ** 2 + dx[None, :] ** 2) / 2.0 / r)
            out[iz, ix] = np.sum(w * g[z0:z1, x0:x1]) / np.sum(w)
    return out


def _bell1d_ref(g, r, axis):
    g = np.moveaxis(g.astype(np.float64), axis, -1)
    n = g.shape[-1]
    out = np.zeros_like(g)
    for p in range(n):
        lo, hi = max(0, p - r), min(n, p + r + 1)
        w = np.exp(-((np.arange(lo, hi) - p) ** 2) / 2.0 / r)
        out[..., p] = (g[..., lo:hi] * w).sum(-1) / w.sum()
    return np.moveaxis(out, -1, axis)


def test_bell_smooth_2d_equals_the_reference_window(ertm):
    g = np.random.default_rng(6).standard_normal((23, 1, 31)).astype(np.float32)
    for r in (1, 3, 8):
        out = ertm.bell_smooth(g, r, ertm.AXIS_X | ertm.AXIS_Z)
        assert np.allclose(out[:, 0], _bell2d_ref(g[:, 0].astype(np.float64), r), atol=2e-6)


def test_bell_smooth_single_axes_and_3d(ertm):
    g = np.random.default_rng(7).standard_normal((9, 7, 11)).astype(np.float32)
    for axes, ax in ((ertm.AXIS_Z, 0), (ertm.AXIS_Y, 1), (ertm.AXIS_X, 2)):
        assert np.allclose(ertm.bell_smooth(g, 2, axes), _bell1d_ref(g, 2, ax), atol=2e-6)
    ref = _bell1d_ref(_bell1d_ref(_bell1d_ref(g, 3, 0), 3, 1), 3, 2)
    assert np.allclose(ertm.bell_smooth(g, 3, 7), ref, atol=3e-6)
    lib = ertm.lib()
    assert lib.ertm_bell_smooth(g.ctypes.data, g.ctypes.data, None, 11, 7, 9, 0, 1, None) == -1
    assert lib.ertm_bell_smooth(g.ctypes.data, g.ctypes.data, None, 11, 7, 9, 65, 1, None) == -1
    assert lib.ertm_bell_smooth(g.ctypes.data, g.ctypes.data, None, 11, 7, 9, 2, 3, None) == -1  # no work


def _taper_ref(nx, left, right, power):
    ix = np.arange(nx, dtype=np.float64)
    f = np.ones(nx)
    if left:
        m = ix <= left
        f[m] *= np.cos(np.pi / 2 * (left - ix[m]) / left) ** power
    if right:
        m = ix >= nx - right
        f[m] *= np.cos(np.pi / 2 * (ix[m] - nx + right) / right) ** power
    return f


def test_taper_x(ertm):
    g = np.random.default_rng(8).standard_normal((5, 2, 40)).astype(np.float32)
    out = ertm.taper_x(g.copy(), 10, 6, 3)
    assert np.allclose(out, g * _taper_ref(40, 10, 6, 3), rtol=1e-6, atol=1e-7)
    assert np.all(out[..., 0] == 0)
    assert np.array_equal(ertm.taper_x(g.copy(), 0, 0, 3), g)


@pytest.mark.gpu
def test_post_filters_on_the_device_match_the_host(ertm):
    import torch
    g = np.random.default_rng(9).standard_normal((70, 33, 90)).astype(np.float32)
    d = torch.from_numpy(g).cuda()
    for r, axes in ((4, ertm.AXIS_X | ertm.AXIS_Z), (2, 7), (5, ertm.AXIS_Y)):
        host = ertm.bell_smooth(g, r, axes)
        dev = ertm.bell_smooth(d, r, axes).cpu().numpy()
        assert np.allclose(dev, host, rtol=1e-6, atol=1e-6)
    host = ertm.taper_x(g.copy(), 20, 13, 3)
    dev = ertm.taper_x(d.clone(), 20, 13, 3).cpu().numpy()
    assert np.allclose(dev, host, rtol=1e-6, atol=1e-7)
    host = ertm.aperture_taper(g.copy(), 15, 70, 6, 2)
    dev = ertm.aperture_taper(d.clone(), 15, 70, 6, 2).cpu().numpy()
    assert np.allclose(dev, host, rtol=1e-6, atol=1e-7)


def _gold():
    import json
    import os
    return json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_helpers.json")))


def _ix_major_to_vol(v, nx, nz):
    return np.asarray(v, np.float32).reshape(nx, nz).T.copy()[:, None, :]


def test_laplace_filter_matches_the_reference_cpu_laplace(ertm):
    """Golden vectors from the reference's own cpu_laplace (12 x 9 image).  Every
    cell agrees except the reference's row-copy quirk: it copies the top and bottom
    rows only for columns 0..nz-1 and its corner copies read a raw -r value; those
    cells hold -r v^2/4 (uncopied) or the corner value in the reference."""
    G = _gold()
    nx, nz = 12, 9
    img = _ix_major_to_vol(G["laplace_in_ix_major"], nx, nz)
    vel = _ix_major_to_vol(G["laplace_vel_ix_major"], nx, nz)
    ref = _ix_major_to_vol(G["laplace_out_ix_major"], nx, nz)
    out = ertm.laplace_filter(img, vel, (5.0, 5.0, 4.0))
    quirk = np.zeros((nz, 1, nx), bool)
    quirk[[0, nz - 1], 0, 0] = True
    quirk[[0, nz - 1], 0, nz:] = True
    scale = np.abs(ref).max()
    assert np.allclose(out[~quirk], ref[~quirk], rtol=1e-5, atol=1e-6 * scale)
    # uncopied row cells keep -r v^2/4; the last column then copies its neighbour's -r
    for k in (0, nz - 1):
        assert np.allclose(ref[k, 0, nz:nx - 1], -img[k, 0, nz:nx - 1] * vel[k, 0, nz:nx - 1] ** 2 / 4, rtol=1e-6)
        assert np.isclose(ref[k, 0, nx - 1], -img[k, 0, nx - 2] * vel[k, 0, nx - 1] ** 2 / 4, rtol=1e-6)


@pytest.mark.parametrize("nz", [15, 16])
def test_hilbert_matches_the_reference_suhilbt(ertm, nz):
    """Golden vectors from the reference's own suhilbt (5 columns); the reference
    accumulates its spectrum in float, this library in double."""
    G = _gold()
    nx = 5
    img = _ix_major_to_vol(G[f"hilbert_in_nz{nz}_ix_major"], nx, nz)
    ref = _ix_major_to_vol(G[f"hilbert_out_nz{nz}_ix_major"], nx, nz)
    out = ertm.hilbert_z(img)
    assert np.allclose(out, ref, rtol=0, atol=2e-5 * np.abs(ref).max())


def _aperture_ref(g, offset_left, offset_right, receiver_offset, offset_attenuation):
    """cauda_zero_and_attenuation_truncation (viscoelastic_equation.cu:2928-2988) restated
    column by column."""
    g = g.astype(np.float64).copy()
    nx = g.shape[-1]
    for ix in range(nx):
        col = g[..., ix]
        if offset_left > receiver_offset:
            if 0 <= ix < offset_left - receiver_offset:
                col[...] = 0
            dl = receiver_offset // offset_attenuation
            dl = 3 if dl <= 2 else dl
            if offset_left - receiver_offset <= ix < offset_left - receiver_offset + dl and offset_left != 0:
                m = offset_left - receiver_offset + dl - ix
                col *= np.cos(np.pi / 2 * m / dl) ** 2
        if offset_right > receiver_offset:
            if offset_left + receiver_offset <= ix < nx:
                col[...] = 0
            dr = receiver_offset // offset_attenuation
            dr = 3 if dr <= 2 else dr
            if offset_left + receiver_offset - dr <= ix < offset_left + receiver_offset and offset_right != 0:
                m = ix - (offset_left + receiver_offset - dr)
                col *= np.cos(np.pi / 2 * m / dr) ** 2
    return g


@pytest.mark.parametrize("ol,orr,ro,oa", [(60, 70, 25, 5), (20, 90, 25, 5), (60, 10, 25, 20), (60, 70, 8, 4)])
def test_aperture_taper_matches_the_reference_kernel(ertm, ol, orr, ro, oa):
    g = np.random.default_rng(15).standard_normal((6, 1, 130)).astype(np.float32)
    w = max(3, ro // oa)
    x0 = ol - ro if ol > ro else -1
    x1 = ol + ro if orr > ro else -1
    out = ertm.aperture_taper(g.copy(), x0, x1, w, 2)
    assert np.allclose(out, _aperture_ref(g, ol, orr, ro, oa), rtol=1e-5, atol=1e-7)
