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


def test_run_log_records_pass_calls(tmp_path):
    """The per-call JSON-lines log of Context (driven here by a stand-in object, no GPU)."""
    import json
    ertm = importlib.import_module(PKG)

    class Fake:
        cfg = ertm.Config(nx=10, ny=1, nz=8, dx=5.0, dy=5.0, dz=5.0, dt_ms=0.5, nt=30, src_steps=20)
        ncell = 80

        @ertm._logged
        def rtm_shot(self, x):
            return x * 2

        @ertm._logged
        def born_adjoint(self):
            return None

    f = Fake()
    assert f.rtm_shot(3) == 6                  # no log set: plain call
    f._log = str(tmp_path / "run.jsonl")
    f.rtm_shot(4)
    f.born_adjoint()
    recs = [json.loads(x) for x in open(f._log)]
    assert [r["call"] for r in recs] == ["rtm_shot", "born_adjoint"]
    assert recs[0]["cell_steps"] == 80 * (20 + 30) and recs[1]["cell_steps"] == 80 * 90
