"""Seeded synthetic models, wavelets and acquisition for the documented workloads.

No public dataset is involved: every model is generated here from a seed.
All volumes are float32 numpy arrays shaped (nz, ny, nx), x fastest, and
include the absorbing layers (the reference's padded nnx/nny/nnz grid).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

BASE_SEED = 20261203


def ricker(freq_hz: float, dt_s: float) -> np.ndarray:
    """Ricker wavelet with the sampling of make_ricker_new (3D_elastic_RTM/zzzzz:139-160):
    Bpar = sqrt(6)/(pi f), N = ceil(1.35 Bpar/dt), 2N+1 samples peaking at sample N,
    w = 0.5 (2 - u^2) exp(-u^2/4), u = 2 sqrt(6) t / Bpar (float32 arithmetic)."""
    f = np.float32(freq_hz if freq_hz else 30.0)
    dt = np.float32(dt_s if dt_s else 0.004)
    bpar = np.float32(math.sqrt(6.0) / (math.pi * float(f)))
    n = int(math.ceil(1.35 * float(bpar) / float(dt)))
    w = np.zeros(2 * n + 1, np.float32)
    w[n] = 1.0
    for i in range(1, n + 1):
        t = np.float32(dt * np.float32(i))
        u = np.float32(2.0 * math.sqrt(6.0) * float(t) / float(bpar))
        uu = float(np.float32(u * u))          # float product, as in the reference
        v = np.float32(0.5 * (2.0 - uu) * math.exp(-uu / 4.0))
        w[n + i] = v
        w[n - i] = v
    return w


def vs_from_vp(vp):
    """Vs = Vp / sqrt(3) (vp_set_vs, 3D_elastic_RTM/zzzzz:1261-1270, double arithmetic
    rounded once to float)."""
    return (np.asarray(vp, np.float32).astype(np.float64) / math.sqrt(3) * 1.0).astype(np.float32)


REFERENCE_GARDNER = 1000 * 0.23   # vp_set_density, 3D_elastic_RTM/zzzzz:1272-1287


def gardner(vp, a: float = 310.0):
    """rho = a * Vp^0.25 in double, rounded once to float.  The reference helper
    vp_set_density uses a = 1000*0.23 (REFERENCE_GARDNER); the workloads use 310."""
    vp = np.asarray(vp, np.float32).astype(np.float64)
    return (a * np.sqrt(np.sqrt(vp))).astype(np.float32)


def pad_edges(v: np.ndarray, pads) -> np.ndarray:
    """Edge-replicating padding of a (nz, ny, nx) volume by (z0, z1, y0, y1, x0, x1)
    cells, the model extension of add_pml_layers_v_h (3D_elastic_RTM/3D_zzzzz:141-259)."""
    z0, z1, y0, y1, x0, x1 = pads
    return np.pad(v, ((z0, z1), (y0, y1), (x0, x1)), mode="edge").astype(np.float32)


def gaussian_smooth(v: np.ndarray, sigma_cells: float, device: str | None = None) -> np.ndarray:
    """Separable Gaussian smoothing (sigma in cells, truncated at 4 sigma, edge-replicated),
    used to build migration models.  Runs on a GPU through torch when one is present."""
    import torch
    if sigma_cells <= 0:
        return v.copy()
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    r = int(math.ceil(4 * sigma_cells))
    x = torch.arange(-r, r + 1, dtype=torch.float64)
    k = torch.exp(-0.5 * (x / sigma_cells) ** 2)
    k = (k / k.sum()).to(torch.float32).to(device)
    t = torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(device)
    for axis in range(3):
        if t.shape[axis] == 1:
            continue
        t = t.movedim(axis, -1)
        shp = t.shape
        flat = t.reshape(-1, 1, shp[-1])
        flat = torch.nn.functional.pad(flat, (r, r), mode="replicate")
        flat = torch.nn.functional.conv1d(flat, k.view(1, 1, -1))
        t = flat.reshape(shp).movedim(-1, axis)
    return t.cpu().numpy().astype(np.float32)


@dataclass
class Workload:
    name: str
    shape: tuple           # (nz, ny, nx) incl. absorbing layers
    dx: float
    dy: float
    dz: float
    dt_ms: float
    nt: int
    pml: int
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    svp: np.ndarray
    svs: np.ndarray
    srho: np.ndarray
    freq: float
    src: tuple             # (sx, sy, sz) cell
    rec: dict              # rx0, nrx, drx, ry0, nry, dry, rz


def layered_2d(seed: int = BASE_SEED, smooth: bool = True) -> Workload:
    """2D workload: 600 x 300 interior at 5 m plus a 40-cell absorbing frame (680 x 380);
    three flat layers with tops at 0/500/1000 m and Vp 1800/2500/3200 m/s, Vs = Vp/sqrt(3),
    rho = 310 Vp^0.25, a +10 % Gaussian lens on Vp and Vs (sigma 40 m at x 1500 m, z 900 m);
    migration model smoothed with sigma 10 cells; dt 0.5 ms, nt 3000, 15 Hz Ricker at
    (1500 m, 25 m), 600 receivers at z = 25 m."""
    nxi, nzi, h, pml = 600, 300, 5.0, 40
    z = (np.arange(nzi) + 0.5) * h
    x = (np.arange(nxi) + 0.5) * h
    vp1 = np.where(z < 500, 1800.0, np.where(z < 1000, 2500.0, 3200.0))
    vp = np.repeat(vp1[:, None], nxi, axis=1)
    X, Z = np.meshgrid(x, z)
    lens = 1.0 + 0.10 * np.exp(-((X - 1500) ** 2 + (Z - 900) ** 2) / (2 * 40.0 ** 2))
    vs = vp / math.sqrt(3) * lens
    vp = vp * lens
    rho = gardner(vp)
    pads = (pml, pml, 0, 0, pml, pml)
    vp, vs, rho = (pad_edges(a.astype(np.float32)[:, None, :], pads) for a in (vp, vs, rho))
    if smooth:
        svp, svs, srho = (gaussian_smooth(a, 10.0) for a in (vp, vs, rho))
    else:
        svp, svs, srho = vp.copy(), vs.copy(), rho.copy()
    nx = nxi + 2 * pml
    rz = pml + int(round(25.0 / h))
    return Workload("2d-layered-lens-680x380", vp.shape, h, h, h, 0.5, 3000, pml, vp, vs, rho,
                    svp, svs, srho, 15.0, (pml + int(round(1500 / h)), 0, rz),
                    dict(rx0=pml, nrx=nxi, drx=1, ry0=0, nry=1, dry=1, rz=rz))


def layered_3d(n_interior=(300, 400, 400), h: float = 10.0, pml: int = 40, nt: int = 4000,
               dt_ms: float = 0.8, seed: int = BASE_SEED, smooth_sigma: float = 8.0,
               rec_every: int = 2) -> Workload:
    """3D workload: interior nz x ny x nx = 300 x 400 x 400 at 10 m with a 40-cell
    absorbing frame (380 x 480 x 480 = 87.55 M cells); five flat layers with seeded tops and
    Vp 2000..3800 m/s, Vs = Vp/sqrt(3), Gardner density (310 Vp^0.25); an ellipsoidal body
    (Vp 4500, Vs 2600, rho 2150, semi-axes 800/600/400 m); migration model smoothed with
    sigma 8 cells; 10 Hz Ricker at the surface centre; receivers every 2 cells (20 m) on the
    whole surface (200 x 200); dt 0.8 ms, nt 4000."""
    nzi, nyi, nxi = n_interior
    rng = np.random.default_rng(seed)
    depth = nzi * h
    tops = np.sort(rng.uniform(0.1 * depth, 0.9 * depth, size=4))
    vps = np.linspace(2000.0, 3800.0, 5)
    z = (np.arange(nzi) + 0.5) * h
    layer = np.searchsorted(tops, z)
    vp1 = vps[layer].astype(np.float32)
    vp = np.broadcast_to(vp1[:, None, None], (nzi, nyi, nxi)).astype(np.float32).copy()
    vs = vs_from_vp(vp)
    rho = gardner(vp)
    zc, yc, xc = 0.6 * depth, 0.5 * nyi * h, 0.5 * nxi * h
    Z = ((np.arange(nzi) + 0.5) * h - zc)[:, None, None]
    Y = ((np.arange(nyi) + 0.5) * h - yc)[None, :, None]
    X = ((np.arange(nxi) + 0.5) * h - xc)[None, None, :]
    body = (X / 800.0) ** 2 + (Y / 600.0) ** 2 + (Z / 400.0) ** 2 <= 1.0
    vp[body], vs[body], rho[body] = 4500.0, 2600.0, 2150.0
    pads = (pml,) * 6
    vp, vs, rho = (pad_edges(a, pads) for a in (vp, vs, rho))
    if smooth_sigma > 0:
        svp, svs, srho = (gaussian_smooth(a, smooth_sigma) for a in (vp, vs, rho))
    else:
        svp, svs, srho = vp.copy(), vs.copy(), rho.copy()
    nz, ny, nx = vp.shape
    sz = pml + 2
    nrx = (nxi + rec_every - 1) // rec_every
    nry = (nyi + rec_every - 1) // rec_every
    return Workload(f"3d-layered-ellipsoid-{nx}x{ny}x{nz}", vp.shape, h, h, h, dt_ms, nt, pml,
                    vp, vs, rho, svp, svs, srho, 10.0, (nx // 2, ny // 2, sz),
                    dict(rx0=pml, nrx=nrx, drx=rec_every, ry0=pml, nry=nry, dry=rec_every, rz=sz))


def windows_3d(nshots: int = 64, seed: int = BASE_SEED + 3, n_interior=(200, 256, 256),
               wmin: int = 64, wmax: int = 192, ntmin: int = 2000, ntmax: int = 3500,
               pml: int = 40, rec_every: int = 2, smooth_sigma: float = 8.0):
    """Batched-window workload: a shared 256 x 256 x 200 model at 10 m (layered plus
    ellipsoid, generated as `layered_3d`) and `nshots` seeded shots, each on its own
    aperture window of wx x wy ~ U[wmin, wmax] cells centred on a random source
    position (shifted to fit the model), nt ~ U[ntmin, ntmax] at 0.8 ms, 10 Hz Ricker
    at 20 m depth and receivers every `rec_every` cells over the window.  Returns
    (migration model (vp, vs, rho), windows as dicts, shots as dicts); the absorbing
    frame of `pml` cells is added around every window by the batched driver."""
    wl = layered_3d(n_interior=n_interior, pml=0, nt=1, smooth_sigma=smooth_sigma)
    nz, ny, nx = n_interior
    rng = np.random.default_rng(seed)
    wins, shots = [], []
    for _ in range(nshots):
        wx, wy = (int(v) for v in rng.integers(wmin, wmax + 1, size=2))
        cx, cy = int(rng.integers(0, nx)), int(rng.integers(0, ny))
        x0 = min(max(cx - wx // 2, 0), nx - wx)
        y0 = min(max(cy - wy // 2, 0), ny - wy)
        nt = int(rng.integers(ntmin, ntmax + 1))
        wins.append(dict(x0=x0, y0=y0, wx=wx, wy=wy, nt=nt))
        shots.append(dict(sx=min(max(cx, x0), x0 + wx - 1), sy=min(max(cy, y0), y0 + wy - 1), sz=2,
                          rx0=x0, nrx=(wx + rec_every - 1) // rec_every, drx=rec_every,
                          ry0=y0, nry=(wy + rec_every - 1) // rec_every, dry=rec_every, rz=2))
    return (wl.svp, wl.svs, wl.srho), wins, shots


def faulted_2d(seed: int, nz: int = 400, nx: int = 800, h: float = 5.0, vmin: float = 1800.0,
               vmax: float = 4000.0):
    """2D layered-and-faulted model (the LSRTM workload's generator): 8-12 layers with
    seeded tops and Vp increasing with depth in [vmin, vmax], cut by 2-4 dipping normal
    faults (dip 50-70 degrees, throw 20-80 m, hanging wall down); Vs = Vp/sqrt(3),
    density 310 Vp^0.25.  Returns (vp, vs, rho), each (nz, 1, nx) float32."""
    rng = np.random.default_rng(seed)
    nl = int(rng.integers(8, 13))
    depth = nz * h
    tops = np.sort(rng.uniform(0.05 * depth, 0.95 * depth, size=nl - 1))
    vps = np.sort(rng.uniform(vmin, vmax, size=nl))
    z = (np.arange(nz) + 0.5) * h
    x = (np.arange(nx) + 0.5) * h
    Z = np.broadcast_to(z[:, None], (nz, nx)).copy()
    for _ in range(int(rng.integers(2, 5))):
        x0 = rng.uniform(0.15, 0.85) * nx * h
        dip = np.deg2rad(rng.uniform(50.0, 70.0)) * rng.choice([-1.0, 1.0])
        throw = rng.uniform(20.0, 80.0)
        # the fault plane x = x0 + z / tan(dip); cells on the hanging-wall side sample
        # the layering `throw` shallower (their layers moved down)
        side = (x[None, :] - (x0 + Z / np.tan(dip))) * np.sign(dip) > 0
        Z = np.where(side, Z - throw, Z)
    layer = np.searchsorted(tops, Z)
    vp = vps[layer].astype(np.float32)[:, None, :]
    vs = vs_from_vp(vp)
    rho = gardner(vp)
    return vp, vs, rho
