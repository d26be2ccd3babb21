"""File formats of the reference and the direct-wave mute (host code, no GPU)."""
import os

import numpy as np
import pytest


def test_volume_round_trip_in_the_reference_order(ertm, tmp_path):
    rng = np.random.default_rng(0)
    v = rng.standard_normal((7, 5, 6)).astype(np.float32)        # (nz, ny, nx)
    p = str(tmp_path / "vol.bin")
    ertm.write_volume_xyz(p, v)
    raw = np.fromfile(p, np.float32)
    # x outer, z inner: file index ((ix * ny) + iy) * nz + iz
    assert np.array_equal(raw, v.transpose(2, 1, 0).ravel())
    assert np.array_equal(ertm.read_volume_xyz(p, 6, 5, 7), v)


def test_cut_boundary_variants(ertm, tmp_path):
    rng = np.random.default_rng(1)
    padded = rng.standard_normal((12, 9, 14)).astype(np.float32)
    p = str(tmp_path / "cut.bin")
    # interior 6 x 5 x 7 at offsets bl=3, bf=2, bu=4 (output_file_xyz_boundary)
    ertm.write_volume_xyz(p, padded, cut=(6, 5, 7, 3, 2, 4))
    inner = padded[4:11, 2:7, 3:9]
    assert np.array_equal(np.fromfile(p, np.float32), inner.transpose(2, 1, 0).ravel())
    back = np.zeros_like(padded)
    ertm.read_volume_xyz(p, 6, 5, 7, into=back, offsets=(3, 2, 4))
    assert np.array_equal(back[4:11, 2:7, 3:9], inner)
    assert not back[:4].any() and not back[11:].any()


def test_shot_gather_files(ertm, tmp_path):
    d = np.random.default_rng(2).standard_normal((3, 11, 4)).astype(np.float32)
    pre = str(tmp_path / "obs_shot")
    ertm.write_shot_gathers(pre, d)
    assert np.array_equal(np.fromfile(pre + "_z.bin", np.float32).reshape(4, 11), d[2].T)
    assert np.array_equal(ertm.read_shot_gathers(pre, 11, 4), d)


def test_direct_wave_mute_matches_its_definition(ertm):
    nt, dt_ms, h, v = 200, 1.0, (10.0, 10.0, 5.0), 2000.0
    w = np.ones(12, np.float32)
    shot = ertm.Shot(20, 3, 4, wavelet=w, rx0=5, nrx=9, drx=4, ry0=1, nry=3, dry=2, rz=2)
    d = np.ones((3, nt, shot.nrec), np.float32)
    ertm.mute_direct(shot, d, dt_ms, h, v, extra=5)
    for r in range(shot.nrec):
        rx, ry = 5 + (r % 9) * 4, 1 + (r // 9) * 2
        dist = np.sqrt(((rx - 20) * h[0]) ** 2 + ((ry - 3) * h[1]) ** 2 + ((2 - 4) * h[2]) ** 2)
        m = int(np.ceil(np.float32(dist) / np.float32(v) / np.float32(dt_ms / 1000))) + 12 + 5
        assert not d[:, :m, r].any() and d[:, m:, r].all(), r


@pytest.mark.gpu
def test_direct_wave_mute_on_the_device_matches_the_host(ertm):
    import torch
    w = np.ones(9, np.float32)
    shot = ertm.Shot(30, 0, 3, wavelet=w, rx0=0, nrx=64, drx=1, rz=3)
    d = np.random.default_rng(3).standard_normal((3, 300, 64)).astype(np.float32)
    host = ertm.mute_direct(shot, d.copy(), 0.5, (5.0, 5.0, 5.0), 1800.0, extra=3)
    dev = torch.from_numpy(d).cuda()
    ertm.mute_direct(shot, dev, 0.5, (5.0, 5.0, 5.0), 1800.0, extra=3)
    assert np.array_equal(dev.cpu().numpy(), host)



def test_reference_output_file_sets(ertm, tmp_path):
    """Per-shot images and excitation arrays under the reference's file names, cut
    to the interior, x-outer (output_3d_result / output_3d_wavefiled_excitation_amp_time)."""
    cfg = ertm.Config(nx=14, ny=9, nz=11, dx=10, dy=10, dz=10, dt_ms=1, nt=10, pml=(3, 2, 1, 2, 4, 1))
    shot = ertm.Shot(7, 4, 5, wavelet=[1.0])
    rng = np.random.default_rng(3)
    pp, ps, tp = (rng.standard_normal(cfg.shape).astype(np.float32) for _ in range(3))
    paths = ertm.write_shot_results(str(tmp_path), cfg, shot, pp, ps, tp)
    assert [os.path.basename(p) for p in paths] == ["result-tp-3-4", "result-pp-3-4", "result-ps-3-4"]
    nxi, nyi, nzi = 14 - 5, 9 - 3, 11 - 5
    back = ertm.read_volume_xyz(paths[1], nxi, nyi, nzi)
    assert np.array_equal(back, pp[4:4 + nzi, 1:1 + nyi, 3:3 + nxi])
    raw = np.fromfile(paths[0], np.float32).reshape(nxi, nyi, nzi)          # x-outer, z-inner
    assert np.array_equal(raw, tp[4:4 + nzi, 1:1 + nyi, 3:3 + nxi].transpose(2, 1, 0))
    vsp = ertm.write_shot_results(str(tmp_path), cfg, shot, pp, ps, tp, vsp=True, prefix="compensate-result")
    assert os.path.basename(vsp[2]) == "compensate-result-ps-1"
    ex = {"time": rng.integers(0, 9, cfg.shape).astype(np.int32),
          **{k: rng.standard_normal(cfg.shape).astype(np.float32) for k in ("amp", "etp", "evx", "evy", "evz")}}
    files = ertm.write_excitation_files(str(tmp_path), cfg, shot, ex)
    names = [os.path.basename(f) for f in files]
    assert names[0] == "ex-time-3-4" and "cut-ex-vzp-3-4" in names
    full = ertm.read_volume_xyz(files[0], 14, 9, 11)
    assert np.array_equal(full, ex["time"].astype(np.float32))
    amp = ertm.read_volume_xyz(os.path.join(str(tmp_path), "cut-ex-amp-3-4"), nxi, nyi, nzi)
    assert np.array_equal(amp, ex["amp"][4:4 + nzi, 1:1 + nyi, 3:3 + nxi])
