"""The post-imaging products against the reference's own 2D CUDA kernels (CPU).

tests/golden/ref_kernels_2d_post.npz holds outputs of the reference's kernels,
compiled from its tree and run once on a B200 by
tests/golden/make_golden_kernels.py on seeded inputs:
  * sum_poynting + caculate_ex_angle_pp_only_RTM (5 x 5 window) and
    caculate_ex_angle_rp_only_RTM (9 x 9) — 2D_elastic_RTM/elastic_2D_kernel_2.cu:8-30,
    elastic_2D_kernel_3.cu:132-284: pins the oracle's angle restatement;
  * imaging_pp/ps_compensate_dependent_angle_2D and the sign variants
    (elastic_2D_kernel_3.cu:622-761): pins ertm_angle_compensate;
  * cuda_bell_smoothz_new / _x_new / _2d (viscoelastic_equation.cu:2528-2604): pins
    ertm_bell_smooth (the 2D window factors into a z pass and an x pass);
  * cuda_attenuation_truncation / cauda_zero_and_attenuation_truncation
    (viscoelastic_equation.cu:2881-2988): pins ertm_taper_x / ertm_aperture_taper.
The library's functions run on the host here.  Tolerances are float rounding: the
reference evaluates exp, cos and pow in float on the GPU, the host code in double.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "ref_kernels_2d_post.npz")


@pytest.fixture(scope="module")
def fx():
    if not os.path.exists(FIX):
        pytest.fail("tests/golden/ref_kernels_2d_post.npz is missing: run "
                    "tests/golden/make_golden_kernels.py --post on a GPU")
    return np.load(FIX)


@pytest.mark.parametrize("name,hw", [("ang_pp", 2), ("ang_rp", 4)])
def test_oracle_angle_matches_reference_kernel(orc, fx, name, hw):
    nx, nz, it = (int(v) for v in fx["ang_meta"])
    got = orc.angle_given(fx["ang_tp"], fx["ang_vxp"], fx["ang_vzp"], fx["ang_time"], it, hw,
                          init=-999.0)
    ref = fx[name]
    written = ref != -999.0
    assert np.array_equal(got != -999.0, written)           # same cells written, same skipped
    assert written.sum() > 100 and (~written & (fx["ang_time"] == it)).sum() > 0
    assert np.abs(got[written] - ref[written]).max() <= 2e-5   # degrees


def test_receiver_window_is_wider_than_source_window(fx):
    """The reference's two angle kernels differ only in the window; the fixtures show it."""
    w = (fx["ang_pp"] != -999.0) & (fx["ang_rp"] != -999.0)
    assert np.abs(fx["ang_pp"][w] - fx["ang_rp"][w]).max() > 1.0


@pytest.mark.parametrize("kind", range(4))
def test_angle_compensation_matches_reference_kernel(ertm, fx, kind):
    got = ertm.angle_compensate(fx["comp_img"], fx["comp_src"], fx["comp_rcv"], kind)
    ref = fx[f"comp_out{kind}"]
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-7)


def test_compensation_open_angle(fx):
    # the reference's first two kernels also rewrite the receiver angle with the open angle
    for kind in (0, 1):
        np.testing.assert_array_equal(fx[f"comp_open{kind}"], fx["comp_src"] - fx["comp_rcv"])


@pytest.mark.parametrize("name,axes,rb", [("bell_z5", "z", 5), ("bell_x5", "x", 5),
                                          ("bell_2d3", "zx", 3)])
def test_bell_smoothing_matches_reference_kernel(ertm, fx, name, axes, rb):
    g = fx["bell_in"][:, None, :]
    ax = (ertm.AXIS_Z if "z" in axes else 0) | (ertm.AXIS_X if "x" in axes else 0)
    got = ertm.bell_smooth(g, rb, ax)[:, 0, :]
    np.testing.assert_allclose(got, fx[name], rtol=2e-5, atol=2e-6)


@pytest.mark.parametrize("name", ["trunc_a", "trunc_b", "trunc_c"])
def test_taper_and_aperture_match_reference_kernel(ertm, fx, name):
    zm, ol, orr, ro, oa = (int(v) for v in fx[name + "_args"])
    g = fx["trunc_in"][:, None, :].copy()
    if zm == 0:
        # cuda_attenuation_truncation: cos^3 ramps over offset/3 columns (receiver_offset != 0)
        ertm.taper_x(g, ol // 3, orr // 3, 3)
    else:
        # cauda_zero_and_attenuation_truncation: zero outside [ol - ro, ol + ro), cos^2
        # ramps of max(3, ro / oa) columns inside each closed edge
        w = ro // oa if ro // oa > 2 else 3
        x0 = ol - ro if ol > ro else -1
        x1 = ol + ro if orr > ro else -1
        ertm.aperture_taper(g, x0, x1, w, 2)
    np.testing.assert_allclose(g[:, 0, :], fx[name], rtol=1e-6, atol=1e-7)
