"""The reference's getpar parameters (3D_elastic_modeling_parameter_sh) read into
the library's configuration."""
import importlib
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = "2d_and_3d_elastic_reverse_time_migration_b200"

PAR = """
# a 3D run in the reference's parameter syntax
RTM=1 GPU_switch=1 GPU_N=1 GPU_start=0 exchange_device_bool=0
lt=4000 dt=0.8 freq=10
join_vs=1 join_den=1 join_shot=0 join_wavefield=0 wavefield_interval=100 infile_shot_name=obs
nx=400 ny=400 nz=300 dx=10 dy=10 dz=10
shot_num_x=2 shot_num_y=1 shot_num_z=1 shot_start_x=100 shot_interval_x=200
shot_start_y=200 shot_interval_y=0 shot_start_z=0 shot_interval_z=0
receiver_num_x=200 receiver_num_y=200 receiver_num_z=1 receiver_start_x=0 receiver_interval_x=2
receiver_start_y=0 receiver_interval_y=2 receiver_start_z=0 receiver_interval_z=0
receiver_offset=0 receiver_mark=0
boundary_up=40 boundary_down=40 boundary_left=40 boundary_right=40 boundary_front=40 boundary_back=40
coe_attenuation=150
velocity_multiple=1 smooth_time_vp=0 smooth_time_vs=0 smooth_time_density=0
velocity=vp.bin velocity1=vs.bin density=rho.bin s_velocity=svp.bin s_velocity1=svs.bin s_density=srho.bin
add_receiver_bool=1 cut_direct_wave=30 laplace=1 laplace_compensate=0 vsp=0 vsp_precon=0
precon=0 precon_z1=0 precon_z2=0
"""


def _params():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    return importlib.import_module(PKG + ".params"), importlib.import_module(PKG)


def test_reference_parameters_give_the_run():
    P, ertm = _params()
    s = P.from_par(P.parse_par(PAR))
    c = s.config
    assert (c.nx, c.ny, c.nz) == (480, 480, 380)
    assert c.pml == (40, 40, 40, 40, 40, 40) and c.nt == 4000 and c.dt_ms == 0.8
    assert c.boundary == ertm.BOUNDARY_SPONGE_COS and c.order == 12 and c.coef_kind == ertm.COEF_REFERENCE12
    assert s.shots == [(140, 240, 40), (340, 240, 40)]
    assert s.receivers == dict(rx0=40, nrx=200, drx=2, ry0=40, nry=200, dry=2, rz=40)
    assert s.inject_mode == ertm.INJECT_ADD and s.mute_extra == 30 and s.laplace
    assert s.files["velocity"] == "vp.bin" and s.files["infile_shot_name"] == "obs"
    # a Shot can be built from the setup
    w = [0.0, 1.0, 0.0]
    shot = ertm.Shot(*s.shots[0], wavelet=w, inject_mode=s.inject_mode, **s.receivers)
    assert shot.nrec == 200 * 200


def test_command_line_overrides_and_missing_keys():
    P, ertm = _params()
    par = P.parse_par(PAR)
    par.update(P.parse_par(["ny=1", "boundary_front=9", "vsp=1", "add_receiver_bool=0"]))
    s = P.from_par(par)
    assert s.config.ny == 1 and s.config.pml[2:4] == (0, 0)
    assert s.config.boundary == ertm.BOUNDARY_SPONGE_CUBIC
    assert s.shots[0][1] == 0 and s.mute_extra is None and s.inject_mode == ertm.INJECT_REPLACE
    assert s.receivers["nry"] == 1 and s.receivers["ry0"] == 0
    del par["lt"]
    with pytest.raises(KeyError, match="lt is not set"):
        P.from_par(par)
    bad = P.parse_par(PAR)
    bad["shot_start_x"] = "1000"
    with pytest.raises(ValueError, match="outside"):
        P.from_par(bad)
