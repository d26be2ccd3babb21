"""Propagation angles at the excitation time, angle-dependent compensation and
angle-domain common-image gathers (2D_elastic_RTM/elastic_2D_kernel_3.cu:132-284,
489-511, 622-761; Poynting vectors of elastic_2D_kernel_2.cu:8-30).

The oracle's angle capture is pinned on the CPU against the direction of the
direct P wave of a point source in a homogeneous medium (a known answer), against
a numpy restatement of the 5 x 5 source window applied to the oracle's own
wavefield at the step where a cell's excitation time is set, and (in
test_oracle_ref_post.py) against the reference's own angle kernels.  The GPU path is
then compared with the oracle on the parity case of the imaging tests."""
import numpy as np
import pytest

from _cases import CASES, DT_MS, geometry, model, oracle_grid, product_config

ANGLE_TOL_DEG = 0.5   # GPU vs oracle, per cell, on cells with a clear excitation


def _homogeneous(orc, n=160, src=(80, 50), nsteps=260):
    h, dt = 10.0, 1.0
    g = orc.make_grid(n, 1, n, h, h, h, dt, R=4, boundary=orc.CPML, pml=(20, 20, 0, 0, 20, 20),
                      pml_vmax=3000.0)
    vp = np.full((n, 1, n), 3000, np.float32)
    vs, rho = np.full_like(vp, 1700), np.full_like(vp, 2000)
    shot = orc.make_shot(src[0], 0, src[1], orc.ricker(20.0, dt / 1000))
    return g, (vp, vs, rho), shot


def test_oracle_source_angle_is_the_direct_wave_direction(orc):
    n, (sx, sz) = 160, (80, 50)
    g, (vp, vs, rho), shot = _homogeneous(orc, n, (sx, sz))
    ex = orc.ExcitationArrays((n, 1, n), angles=True)
    orc.run_pass(g, vp, vs, rho, shot, orc.SOURCE, 260, ex=ex)
    k, i = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    dx, dz = i - sx, k - sz
    dist = np.hypot(dx, dz)
    m = (dist >= 20) & (dist < 65) & (np.abs(dz) > 0.5 * np.abs(dx)) & (i > 25) & (i < n - 25) \
        & (k > 25) & (k < n - 25)
    ref = np.degrees(np.arctan(dx[m] / dz[m]))
    err = np.abs(ex.src_angle[:, 0][m] - ref)
    assert m.sum() > 3000
    assert err.max() < 4.0 and np.percentile(err, 90) < 2.0, (err.max(), np.percentile(err, 90))


def _window_angle(f, i, k, hw=2):
    """The reference's window angle (5 x 5 source window, hw = 2), rounded as it rounds:
    float(atan(sxz / szz)) * 180 / 3.1415926f in float."""
    nz, nx = f["tp"].shape[0], f["tp"].shape[2]
    sxz = szz = 0.0
    for kk in range(k - hw, k + hw + 1):
        for ii in range(i - hw, i + hw + 1):
            if 0 <= ii < nx and 0 <= kk < nz:
                tp = float(f["tp"][kk, 0, ii])
                px, pz = -tp * float(f["vxp"][kk, 0, ii]), -tp * float(f["vzp"][kk, 0, ii])
                sxz += px * pz
                szz += pz * pz
    if szz == 0:
        return None
    return float(np.float32(np.arctan(sxz / szz)) * np.float32(180.0) / np.float32(3.1415926))


@pytest.mark.parametrize("nsteps", [90, 130])
def test_oracle_angle_is_the_window_angle_at_the_excitation_step(orc, nsteps):
    n = 80
    g, (vp, vs, rho), shot = _homogeneous(orc, n, (40, 30))
    ex = orc.ExcitationArrays((n, 1, n), angles=True)
    r = orc.run_pass(g, vp, vs, rho, shot, orc.SOURCE, nsteps, ex=ex, want_fields=True)
    cells = np.argwhere(ex.time[:, 0] == nsteps - 1)
    assert len(cells) > 20
    for k, i in cells[:: max(1, len(cells) // 60)]:
        a = _window_angle(r["fields"], i, k)
        assert a is not None
        assert abs(ex.src_angle[k, 0, i] - a) < 1e-4, (k, i)


def _comp_ref(img, s, r, kind):
    d = (s - r).astype(np.float64)
    c, sn = np.cos(np.radians(d)), np.sin(np.abs(np.radians(d)))
    if kind == 0:
        den = np.where((np.abs(d) >= 87.5) & (np.abs(d) <= 92.5), 0.1, c)
        return img / (den + 1e-4)
    if kind == 1:
        den = np.where(np.abs(d) <= 2.5, 0.1, sn)
        return img / (den + 1e-4)
    if kind == 2:
        v = np.where(c <= 0, -img, img)
        return -v / (np.abs(c) + 0.03)
    return -img / (np.abs(np.sin(np.radians(d))) + 0.1)


def test_angle_compensation(ertm):
    rng = np.random.default_rng(12)
    img = rng.standard_normal(4000).astype(np.float32)
    s = rng.uniform(-80, 80, 4000).astype(np.float32)
    r = rng.uniform(-80, 80, 4000).astype(np.float32)
    s[:10], r[:10] = 90.0, 0.0          # open angle in the clamped band
    s[10:20], r[10:20] = 1.0, 0.0       # small open angle (PS clamp)
    for kind in range(4):
        out = ertm.angle_compensate(img, s, r, kind)
        ref = _comp_ref(img.astype(np.float64), s, r, kind)
        assert np.allclose(out, ref, rtol=2e-5, atol=1e-6), kind
    with pytest.raises(ertm.ErtmError):
        ertm.angle_compensate(img, s, r, 4)


def _adcig_ref(img, ang, normal, nang, dangle, sx, zmin, slope):
    nz, nx = img.shape
    cig = np.zeros((2 * nang + 1, nz, nx))
    for iz in range(nz):
        for ix in range(nx):
            if not (iz > zmin and iz > slope * (ix - sx) and iz > slope * (sx - ix)):
                continue
            a = float(np.float32(ang[iz, ix] - (normal[iz, ix] if normal is not None else 0)))
            rr = int((abs(a) + 0.5) / dangle)
            if rr < nang:
                cig[nang + rr if a >= 0 else nang - rr, iz, ix] += img[iz, ix]
    return cig


def test_adcig_binning(ertm):
    rng = np.random.default_rng(13)
    nz, nx = 70, 90
    img = rng.standard_normal((nz, nx)).astype(np.float32)
    ang = rng.uniform(-70, 70, (nz, nx)).astype(np.float32)
    normal = rng.uniform(-5, 5, (nz, nx)).astype(np.float32)
    cig = ertm.adcig_bin(img, ang, 30, 2.0, 40, zmin=10, slope=1.2)
    assert np.allclose(cig, _adcig_ref(img, ang, None, 30, 2.0, 40, 10, 1.2), atol=1e-6)
    cig = ertm.adcig_bin(img, ang, 30, 2.0, 40, zmin=10, slope=1.2, normal=normal, cig=cig)
    ref = _adcig_ref(img, ang, None, 30, 2.0, 40, 10, 1.2) + _adcig_ref(img, ang, normal, 30, 2.0, 40, 10, 1.2)
    assert np.allclose(cig, ref, atol=1e-5)
    # every kept cell (iz > 0 with slope 0) lands in exactly one bin
    full = ertm.adcig_bin(img, np.zeros_like(ang), 5, 2.0, 40, zmin=-1, slope=0.0)
    assert np.allclose(full.sum(0)[1:], img[1:]) and not full[:, 0].any()


def _gpu_and_oracle_angles(ertm, orc):
    case = "2d_r4_cpml"
    c = CASES[case]
    nt, nsrc = 400, 300
    vp, vs, rho = model(c["shape"], seed=7)
    g = oracle_grid(orc, case, vp)
    src, rec = geometry(c["shape"], c["pml"])
    w = orc.ricker(25.0, DT_MS / 1000.0)
    oshot = orc.make_shot(*src, w, **rec)
    data = orc.run_pass(g, vp, vs, rho, oshot, orc.MODEL, nt)["data"]
    ex = orc.ExcitationArrays(c["shape"], angles=True)
    orc.run_pass(g, vp, vs, rho, oshot, orc.SOURCE, nsrc, ex=ex)
    r = orc.run_pass(g, vp, vs, rho, oshot, orc.RECEIVER, nt, data=data, ex=ex)

    ctx = ertm.Context(product_config(ertm, case, nt, nsrc))
    ctx.set_model(ertm.MIGRATION_MODEL, vp, vs, rho)
    ctx.set_angles(True)
    pshot = ertm.Shot(*src, wavelet=w, **rec)
    ctx.forward_together_using_smoothed_model(pshot)
    ctx.backward_together_using_smoothed_model(pshot, data)
    sa, ra = ctx.get_angles()
    gx = ctx.get_excitation()
    clear = (ex.amp2 - ex.second2 > 2e-4 * ex.amp2) & (ex.amp2 > 1e-4 * np.percentile(ex.amp2, 99)) \
        & (gx["time"] == ex.time)
    return ctx, c, ex, r, sa, ra, clear


@pytest.mark.gpu
def test_source_angles_match_the_oracle(ertm, orc):
    ctx, c, ex, _, sa, _, clear = _gpu_and_oracle_angles(ertm, orc)
    assert clear.mean() > 0.5
    d = np.abs(sa - ex.src_angle)[clear]
    assert np.percentile(d, 99) < ANGLE_TOL_DEG and np.median(d) < 0.05, (np.percentile(d, 99), np.median(d))
    ctx.set_angles(False)
    with pytest.raises(ertm.ErtmError):
        ctx.get_angles()
    ctx3 = ertm.Context(product_config(ertm, "3d_r4_cpml", 50))
    with pytest.raises(ertm.ErtmError):
        ctx3.set_angles(True)


@pytest.mark.gpu
def test_receiver_angles_match_the_oracle(ertm, orc):
    """Receiver angles are compared where the receiver window holds a wavefield: at
    about 40 % of the clearly excited cells of this case the back-propagated field
    has not arrived at the excitation step and the window holds only the stencil's
    numerical precursor (P energy 1e-70 of the maximum and below), where the angle
    of float data means nothing (the reference computes it from float Poynting
    arrays too).  Cells above 1e-10 of the largest window energy are compared
    (about 40 % of the clearly excited cells); on them, white noise of 1e-5 of the
    data maximum moves the oracle's angles by 0.04 degrees at the 99th percentile."""
    ctx, c, ex, r, _, ra, clear = _gpu_and_oracle_angles(ertm, orc)
    e = ex.rcv_energy
    live = clear & (e > 1e-10 * e[clear].max())
    assert live.sum() > 0.25 * clear.sum()
    d = np.abs(ra - ex.rcv_angle)[live]
    assert np.percentile(d, 99) < ANGLE_TOL_DEG and np.median(d) < 0.05, (np.percentile(d, 99), np.median(d))


@pytest.mark.gpu
def test_angle_products_on_the_device_match_the_host(ertm):
    import torch
    rng = np.random.default_rng(14)
    shape = (83, 1, 97)
    img = rng.standard_normal(shape).astype(np.float32)
    sa = rng.uniform(-80, 80, shape).astype(np.float32)
    ra = rng.uniform(-80, 80, shape).astype(np.float32)
    dev = [torch.from_numpy(a).cuda() for a in (img, sa, ra)]
    for kind in range(4):
        h = ertm.angle_compensate(img, sa, ra, kind)
        d = ertm.angle_compensate(*dev, kind).cpu().numpy()
        assert np.allclose(d, h, rtol=1e-5, atol=1e-6 * np.abs(h).max()), kind
    h = ertm.adcig_bin(img, sa, 20, 3.0, 48, zmin=5)
    d = ertm.adcig_bin(dev[0], dev[1], 20, 3.0, 48, zmin=5).cpu().numpy()
    assert np.array_equal(d, h)


def test_oracle_receiver_angle_is_the_window_angle_at_the_excitation_step(orc):
    """The receiver pass stepped one step at a time: at each step, the cells whose
    excitation time it is get the 9 x 9 window angle of the receiver wavefield of
    that step (caculate_ex_angle_rp_only_RTM, elastic_2D_kernel_3.cu:209-284)."""
    import ctypes as C
    n, nt, nsrc = 60, 160, 110
    g, (vp, vs, rho), shot = _homogeneous(orc, n, (30, 20))
    rec = orc.make_shot(30, 0, 20, orc.ricker(20.0, 1e-3), rx0=20, nrx=20, drx=1, rz=24)
    data = np.ascontiguousarray(orc.run_pass(g, vp, vs, rho, rec, orc.MODEL, nt)["data"])
    ex = orc.ExcitationArrays((n, 1, n), angles=True)
    orc.run_pass(g, vp, vs, rho, rec, orc.SOURCE, nsrc, ex=ex)
    L = orc.lib()
    st = L.orc_state_create(C.byref(g), orc._fp(vp), orc._fp(vs), orc._fp(rho))
    F = np.zeros((13, n, 1, n), np.float32)
    exs = ex.struct()
    checked = 0
    try:
        for it in range(nt - 1, -1, -1):
            L.orc_state_step(st, C.byref(rec), orc.RECEIVER, it, nt, orc._fp(data), C.byref(exs),
                             None, None, None)
            cells = np.argwhere(ex.time[:, 0] == it)
            if len(cells) == 0 or it % 7:
                continue
            L.orc_state_fields(st, orc._fp(F))
            f = {"tp": F[9], "vxp": F[10], "vzp": F[12]}
            for k, i in cells[:: max(1, len(cells) // 5)]:
                a = _window_angle(f, i, k, hw=4)      # the receiver kernel's 9 x 9 window
                if a is None:
                    continue
                assert abs(ex.rcv_angle[k, 0, i] - a) < 1e-4, (it, k, i)
                checked += 1
    finally:
        L.orc_state_destroy(st)
    assert checked > 20
