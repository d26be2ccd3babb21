"""Pin the oracle (and the product's host helpers) to the reference's own code.

tests/golden/ref_helpers.json holds outputs of the reference's CPU helpers
(3D_elastic_RTM/zzzzz, 3D_elastic_RTM/3D_zzzzz) compiled from the reference
tree by tests/golden/make_golden.py.  Comparisons are bit-exact.
"""
import json
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_helpers.json")))


@pytest.mark.parametrize("key,freq,dt", [("ricker_10_0.0008", 10.0, 0.0008),
                                          ("ricker_15_0.0005", 15.0, 0.0005),
                                          ("ricker_30_0.001", 30.0, 0.001)])
def test_ricker_bit_exact(orc, synth, key, freq, dt):
    ref = np.array(GOLD[key], np.float32)
    assert np.array_equal(orc.ricker(freq, np.float32(dt)), ref)          # oracle
    assert np.array_equal(synth.ricker(freq, np.float32(dt)), ref)        # product helper


def test_reference12_coefficients(orc):
    ref = np.array(GOLD["coe_optimized12"], np.float32)
    assert np.array_equal(orc.coef_reference12().astype(np.float32), ref)


def test_taylor_coefficients(orc):
    c = orc.coef_taylor(4)
    assert np.allclose(c[1:5], [1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168], rtol=1e-12)
    c2 = orc.coef_taylor(1)
    assert abs(c2[1] - 1.0) < 1e-15


def test_sponge_cubic_2d_bit_exact(orc):
    nx, nz, bu, bd, bl, br = 20, 16, 5, 6, 4, 7
    nxa, nza = bl + nx + br, bu + nz + bd
    ref = np.array(GOLD["att2d_cubic_ix_major"], np.float32).reshape(nxa, nza)
    px = orc.sponge_profile(orc.SPONGE_CUBIC, nxa, bl, br, 200.0).astype(np.float32)
    pz = orc.sponge_profile(orc.SPONGE_CUBIC, nza, bu, bd, 200.0).astype(np.float32)
    mine = (pz[None, :] + px[:, None]).astype(np.float32)
    assert np.array_equal(mine, ref)


def test_sponge_cos_3d_bit_exact(orc):
    nx, ny, nz, bu, bd, bl, br, bf, bb = 9, 8, 7, 3, 4, 5, 3, 2, 4
    nxb, nyb, nzb = nx + bl + br, ny + bf + bb, nz + bu + bd
    ref = np.array(GOLD["att3d_cos_z_major"], np.float32).reshape(nzb, nyb, nxb)
    px = orc.sponge_profile(orc.SPONGE_COS, nxb, bl, br, 150.0).astype(np.float32)
    py = orc.sponge_profile(orc.SPONGE_COS, nyb, bf, bb, 150.0).astype(np.float32)
    pz = orc.sponge_profile(orc.SPONGE_COS, nzb, bu, bd, 150.0).astype(np.float32)
    mine = ((pz[:, None, None] + px[None, None, :]) + py[None, :, None]).astype(np.float32)
    assert np.array_equal(mine, ref)


def test_edge_padding_matches_reference(synth):
    nx, ny, nz, bl, bf, bu = 5, 4, 3, 2, 3, 1
    nxb, nyb, nzb = nx + bl + 2, ny + bf + 1, nz + bu + 2
    ref = np.array(GOLD["pad3d_z_major"], np.float32).reshape(nzb, nyb, nxb)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    core = (1000.0 + 100.0 * k + 10.0 * j + i).astype(np.float32)
    mine = synth.pad_edges(core, (bu, nzb - nz - bu, bf, nyb - ny - bf, bl, nxb - nx - bl))
    assert np.array_equal(mine, ref)


def test_vs_and_density_laws(synth):
    vp = np.array(GOLD["vp_in"], np.float32)
    assert np.array_equal(synth.vs_from_vp(vp), np.array(GOLD["vs_from_vp"], np.float32))
    assert np.array_equal(synth.gardner(vp, synth.REFERENCE_GARDNER),
                          np.array(GOLD["rho_from_vp"], np.float32))
