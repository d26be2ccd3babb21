"""The reference's run parameters, read into this library's configuration.

The reference reads about 55 `key=value` parameters with SU's getpar, from the
command line or a parameter file (elastic_modeling_parameter_input,
3D_elastic_RTM/3D_elastic_modeling_parameter_sh:2-164), and stops with
"<key> is not set!" when one is missing.  `parse_par` reads the same syntax and
`from_par` turns the keys that describe the run into a `Config`, the shot list
and the switches around the passes, so a reference run's parameters drive this
library unchanged.

Conventions taken from the reference:
  * nx, ny, nz are interior sizes; the boundary_* widths are added around them
    (the library's grid includes its absorbing layers);
  * shot and receiver positions are interior cells, offset by boundary_left in
    x, boundary_back in y and boundary_up in z, as the calls of add_source_3D
    and write_or_add_shot_3D_surface_three pass them (bl, bb, bu;
    3D_forward_or_back_together.cu:36, :127);
  * dt is in ms, lt is the number of steps, the source pass runs 2*lt/3 steps
    (:173);
  * damping: coe_attenuation with the reference's 3D cosine profile (2D: cubic),
    12th-order optimised coefficients (radius 6);
  * add_receiver_bool = 1 adds the recorded data in the receiver pass, 0 writes
    it over the field; cut_direct_wave > 0 with vsp = 0 mutes the direct wave
    with that many extra samples (:132-136).
"""
from __future__ import annotations

import shlex
from dataclasses import dataclass, field

from . import (BOUNDARY_SPONGE_COS, BOUNDARY_SPONGE_CUBIC, COEF_REFERENCE12, INJECT_ADD, INJECT_REPLACE,
               Config)

INT_KEYS = ("lt", "nx", "ny", "nz",
            "shot_num_x", "shot_num_y", "shot_num_z", "shot_start_x", "shot_interval_x",
            "shot_start_y", "shot_interval_y", "shot_start_z", "shot_interval_z",
            "receiver_num_x", "receiver_num_y", "receiver_num_z", "receiver_start_x",
            "receiver_interval_x", "receiver_start_y", "receiver_interval_y", "receiver_start_z",
            "receiver_interval_z",
            "boundary_up", "boundary_down", "boundary_left", "boundary_right", "boundary_front",
            "boundary_back", "add_receiver_bool", "cut_direct_wave", "laplace", "vsp")
FLOAT_KEYS = ("dt", "freq", "dx", "dy", "dz", "coe_attenuation")
FILE_KEYS = ("velocity", "velocity1", "density", "s_velocity", "s_velocity1", "s_density",
             "infile_shot_name")


def parse_par(source) -> dict:
    """`key=value` pairs from a list of arguments (a command line) or from the
    text of a parameter file (whitespace-separated, `#` starts a comment).  A key
    given twice keeps its last value, as getpar does."""
    if isinstance(source, str):
        items = []
        for line in source.splitlines():
            line = line.split("#", 1)[0]
            items += shlex.split(line)
    else:
        items = list(source)
    out = {}
    for it in items:
        if "=" not in it:
            continue
        k, v = it.split("=", 1)
        out[k.strip()] = v.strip()
    return out


def _get(par: dict, key: str, kind):
    if key not in par:
        raise KeyError(f"{key} is not set!")
    try:
        return kind(par[key])
    except ValueError:
        raise ValueError(f"{key}={par[key]!r} is not a valid {kind.__name__}") from None


@dataclass
class Setup:
    config: Config
    shots: list                      # (sx, sy, sz) source cells of the padded grid, in order
    receivers: dict                  # Shot keyword arguments for the receiver grid
    freq: float                      # Ricker peak frequency, Hz
    inject_mode: int
    mute_extra: int | None           # direct-wave mute (ertm_mute_direct `extra`), None = off
    laplace: bool                    # Laplacian image filter after migration
    files: dict = field(default_factory=dict)


def from_par(par: dict, device: int = 0) -> Setup:
    g = {k: _get(par, k, int) for k in INT_KEYS}
    f = {k: _get(par, k, float) for k in FLOAT_KEYS}
    two_d = g["ny"] == 1
    bl, br, bf, bb = g["boundary_left"], g["boundary_right"], g["boundary_front"], g["boundary_back"]
    bu, bd = g["boundary_up"], g["boundary_down"]
    if two_d:
        bf = bb = 0
    if g["receiver_num_z"] != 1:
        raise ValueError("receiver_num_z must be 1 (one receiver depth)")
    cfg = Config(nx=g["nx"] + bl + br, ny=g["ny"] + bf + bb, nz=g["nz"] + bu + bd,
                 dx=f["dx"], dy=f["dy"], dz=f["dz"], dt_ms=f["dt"], nt=g["lt"], src_steps=0,
                 order=12, coef_kind=COEF_REFERENCE12,
                 boundary=BOUNDARY_SPONGE_CUBIC if two_d else BOUNDARY_SPONGE_COS,
                 pml=(bl, br, bf, bb, bu, bd), sponge_coef=f["coe_attenuation"], device=device)
    shots = []
    for iz in range(g["shot_num_z"]):
        for iy in range(g["shot_num_y"]):
            for ix in range(g["shot_num_x"]):
                shots.append((g["shot_start_x"] + ix * g["shot_interval_x"] + bl,
                              0 if two_d else g["shot_start_y"] + iy * g["shot_interval_y"] + bb,
                              g["shot_start_z"] + iz * g["shot_interval_z"] + bu))
    # an interval of 0 along an axis with one receiver is the reference's "unused"
    rec = dict(rx0=g["receiver_start_x"] + bl, nrx=g["receiver_num_x"], drx=max(1, g["receiver_interval_x"]),
               ry0=0 if two_d else g["receiver_start_y"] + bb, nry=1 if two_d else g["receiver_num_y"],
               dry=1 if two_d else max(1, g["receiver_interval_y"]), rz=g["receiver_start_z"] + bu)
    for s in shots:
        if not (0 <= s[0] < cfg.nx and 0 <= s[1] < cfg.ny and 0 <= s[2] < cfg.nz):
            raise ValueError(f"shot at cell {s} is outside the {cfg.nx}x{cfg.ny}x{cfg.nz} grid")
    inject = INJECT_ADD if g["add_receiver_bool"] else INJECT_REPLACE
    mute = g["cut_direct_wave"] if (g["vsp"] == 0 and g["cut_direct_wave"] > 0) else None
    files = {k: par[k] for k in FILE_KEYS if k in par}
    return Setup(cfg, shots, rec, f["freq"], inject, mute, bool(g["laplace"]), files)
