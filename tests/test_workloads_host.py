"""Synthetic workload generators and the learned-preconditioner host helpers (CPU)."""
import importlib

import numpy as np

PKG = "2d_and_3d_elastic_reverse_time_migration_b200"


def test_faulted_model_follows_its_recipe():
    syn = importlib.import_module(PKG + ".synthetic")
    vp, vs, rho = syn.faulted_2d(3, nz=120, nx=240, h=5.0)
    assert vp.shape == (120, 1, 240) and vp.dtype == np.float32
    assert 1800.0 <= vp.min() and vp.max() <= 4000.0
    assert 8 <= len(np.unique(vp)) <= 12                      # 8-12 layers
    assert np.allclose(vs, vp / np.sqrt(3.0), rtol=1e-6)
    assert np.allclose(rho, 310.0 * vp.astype(np.float64) ** 0.25, rtol=1e-5)
    # velocity never decreases with depth inside a column (faults shift, not invert)
    assert np.all(np.diff(vp[:, 0, :], axis=0) >= 0)
    # at least one fault: some depth sees different layers across x
    assert any(len(np.unique(vp[k, 0, :])) > 1 for k in range(120))
    # seeded
    assert np.array_equal(vp, syn.faulted_2d(3, nz=120, nx=240, h=5.0)[0])


def test_window_workload_geometry():
    syn = importlib.import_module(PKG + ".synthetic")
    (vp, vs, rho), wins, shots = syn.windows_3d(nshots=64, n_interior=(40, 256, 256), smooth_sigma=0)
    assert vp.shape == (40, 256, 256)
    for w, s in zip(wins, shots):
        assert 64 <= w["wx"] <= 192 and 64 <= w["wy"] <= 192
        assert 0 <= w["x0"] and w["x0"] + w["wx"] <= 256 and 0 <= w["y0"] and w["y0"] + w["wy"] <= 256
        assert 2000 <= w["nt"] <= 3500
        assert w["x0"] <= s["sx"] < w["x0"] + w["wx"] and w["y0"] <= s["sy"] < w["y0"] + w["wy"]
        assert s["rx0"] == w["x0"] and s["drx"] == 2 and (s["nrx"] - 1) * 2 < w["wx"]
    cells = np.mean([(w["wx"] + 80) * (w["wy"] + 80) * 280 for w in wins])
    assert 9e6 < cells < 16e6                                 # ~12.5 M cells per padded window


def test_image_packing_round_trip():
    L = importlib.import_module(PKG + ".learned")
    rng = np.random.default_rng(0)
    m = tuple(rng.standard_normal((61, 1, 93)).astype(np.float32) for _ in range(3))
    img = L.to_image(m)
    assert img.shape == (64, 96, 3) and not img[61:].any() and not img[:, 93:].any()
    back = L.from_image(img, m[0].shape)
    assert all(np.array_equal(a, b) for a, b in zip(back, m))
    assert L.iters_to([0.5, 0.2, 0.009, 0.001], 1e-2) == 3
    assert L.iters_to([0.5, 0.2], 1e-2) is None
