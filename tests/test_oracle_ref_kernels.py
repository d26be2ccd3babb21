"""Pin the oracle's scheme to the reference's own 2D CUDA kernels.

tests/golden/ref_kernels_2d.npz holds inputs and outputs of four reference
kernels (compiled from its tree by oracle/ref_kernels/Makefile and run on a
B200 by tests/golden/make_golden_kernels.py):
  fwd_txxzzxzpp_viscoelastic_and_memory_3parameterization (2D_elastic_RTM/
    viscoelastic_equation.cu:184-325; tao = strain = 1, so the elastic stress
    half-step with sponge damping and the 12th-order optimised stencil),
  decom_new (2D_elastic_RTM/elastic_2D_kernel_2.cu:671-791),
  imaging_inner_product_ex_2D (2D_elastic_RTM/elastic_2D_kernel_3.cu:559-580),
  cuda_cal_dem_parameter_viscoelastic_media_new (2D_elastic_RTM/
    viscoelastic_equation.cu:2398-2505; inversion_para 2).
The oracle computes in double precision from the same float32 inputs, so the
two agree to the float32 rounding of the reference (measured ~1e-7 relative
L2); the bound below is 5e-7.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_kernels_2d.npz")
TOL = 5e-7


def _load():
    d = np.load(GOLD)
    return {k: d[k] for k in d.files}


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


def _grid(orc, d, coef=None):
    nx, nz, rad, dt, dx, sponge = d["meta"][:6]
    pml = [int(v) for v in d["meta"][6:12]]
    return orc.make_grid(int(nx), 1, int(nz), dx, dx, dx, dt, R=int(rad),
                         coef=orc.coef_reference12() if coef is None else coef,
                         boundary=orc.SPONGE_CUBIC, pml=pml, sponge_coef=sponge)


def _stress(orc, d, g):
    return orc.stress_step_given(g, d["vp"], d["vs"], d["rho"],
                                 *[d["in_" + k] for k in ("vx", "vz", "txx", "tzz", "txz")])


def test_fixture_present():
    assert os.path.exists(GOLD)


def test_stress_half_step_matches_reference_kernel(orc):
    d = _load()
    out = _stress(orc, d, _grid(orc, d))
    for o, k in zip(out, ("txx", "tzz", "txz")):
        assert _rel(o, d["stress_" + k]) < TOL, k


def test_stress_comparison_detects_a_different_stencil(orc):
    # the 8th-order weights (zero beyond n = 4) in the same 12-point frame: the
    # comparison must see a change of stencil
    d = _load()
    c8 = np.zeros(7)
    c8[:5] = orc.coef_taylor(4)[:5]
    out = _stress(orc, d, _grid(orc, d, coef=c8))
    assert min(_rel(o, d["stress_" + k]) for o, k in zip(out, ("txx", "tzz", "txz"))) > 100 * TOL


def test_divcurl_matches_decom_new(orc):
    d = _load()
    g = _grid(orc, d)
    col = lambda a: np.ascontiguousarray(a[:, None, :])
    p, _, s, _ = orc.divcurl(g, col(d["vp"]), col(d["vs"]), col(d["in_vx"]), None, col(d["in_vz"]))
    assert _rel(p[:, 0, :], d["decom_p"]) < TOL
    assert _rel(s[:, 0, :], d["decom_s"]) < TOL


def test_imaging_matches_reference_kernel(orc):
    d = _load()
    z = np.zeros_like(d["img_ex"])
    pp, _ = orc.image_given(d["img_ex"], d["img_ez"], d["img_rx"], d["img_rz"], z, z)
    ref = d["img_pp"].ravel()
    ok = np.isfinite(ref)               # the reference divides 0/0 where e == 0
    assert (~ok).sum() == 3 and (pp[~ok] == 0).all()
    assert _rel(pp[ok], ref[ok]) < TOL


def test_born_sources_match_reference_kernel(orc):
    d = _load()
    dt_ms = float(d["meta"][3])
    exz = (d["dem_vx_z"] + d["dem_vz_x"]).astype(np.float32)
    sxx, szz, sxz, svx, svz = orc.born_sources_given(
        dt_ms, d["vp"], d["vs"], d["rho"], d["dem_rvp"], d["dem_rvs"], d["dem_rrho"],
        d["dem_vx_x"], d["dem_vz_z"], exz, d["dem_vx_t"], d["dem_vz_t"])
    assert _rel(sxx, d["dem_sxx"].ravel()) < TOL
    assert _rel(szz, d["dem_szz"].ravel()) < TOL
    assert _rel(sxz, d["dem_sxz"].ravel()) < TOL
    # the reference's velocity source is -drho * v_t with drho the absolute density
    # perturbation; the oracle's is the velocity increment dt * (-drho/rho) * v_t
    rho = d["rho"].ravel().astype(np.float64)
    assert _rel(svx, dt_ms / 1000.0 * d["dem_p1"].ravel() / rho) < TOL
    assert _rel(svz, dt_ms / 1000.0 * d["dem_p2"].ravel() / rho) < TOL
