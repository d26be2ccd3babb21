"""A small batched-window case shared by the window tests: a shared model and
seeded aperture windows, and the per-window reference path (one fresh context
of the window's size per shot, images added on the host)."""
import numpy as np

DT_MS, H, PML = 0.8, 10.0, 10


def shared_model(shape, seed=11):
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    z = np.arange(nz)[:, None, None] * np.ones((1, ny, nx))
    vp = 2000.0 + 25.0 * z
    kz, ky, kx = nz * 0.6, ny * 0.5, nx * 0.5
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    blob = ((zz - kz) / (nz * 0.15)) ** 2 + ((yy - ky) / (ny * 0.25)) ** 2 + ((xx - kx) / (nx * 0.25)) ** 2
    vp = vp + 400.0 * (blob < 1.0) + 5.0 * rng.standard_normal(vp.shape)
    vp = vp.astype(np.float32)
    vs = (vp / np.sqrt(3.0)).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    return vp, vs, rho


def crop_pad(a, x0, y0, wx, wy, pml, two_d):
    """model cropped to the window, all depths, extended by `pml` cells with edge values"""
    nz, ny, nx = a.shape
    iz = np.clip(np.arange(-pml, nz + pml), 0, nz - 1)
    iy = np.array([0]) if two_d else np.clip(np.arange(y0 - pml, y0 + wy + pml), 0, ny - 1)
    ix = np.clip(np.arange(x0 - pml, x0 + wx + pml), 0, nx - 1)
    return np.ascontiguousarray(a[np.ix_(iz, iy, ix)])


def windows(ertm, shape, nshots, seed, two_d, wmin, wmax, ntmin, ntmax):
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    wins, shots = [], []
    wav = None
    for _ in range(nshots):
        wx = int(rng.integers(wmin, wmax + 1))
        wy = 1 if two_d else int(rng.integers(wmin, wmax + 1))
        x0 = int(rng.integers(0, nx - wx + 1))
        y0 = 0 if two_d else int(rng.integers(0, ny - wy + 1))
        nt = int(rng.integers(ntmin, ntmax + 1))
        wins.append(ertm.Window(x0, y0, wx, wy, nt))
        sx, sy = x0 + wx // 2, (0 if two_d else y0 + wy // 2)
        shots.append(dict(sx=sx, sy=sy, sz=2, rx0=x0, nrx=(wx + 1) // 2, drx=2,
                          ry0=y0, nry=1 if two_d else (wy + 1) // 2, dry=2, rz=2))
    return wins, shots


def to_window_shot(ertm, s, w, two_d, wavelet):
    return ertm.Shot(s["sx"] - w.x0 + PML, 0 if two_d else s["sy"] - w.y0 + PML, s["sz"] + PML,
                     wavelet=wavelet, rx0=s["rx0"] - w.x0 + PML, nrx=s["nrx"], drx=s["drx"],
                     ry0=0 if two_d else s["ry0"] - w.y0 + PML, nry=s["nry"], dry=s["dry"],
                     rz=s["rz"] + PML)


def config(ertm, nx, ny, nz, nt, two_d, autotune=0):
    pml = (PML, PML, 0 if two_d else PML, 0 if two_d else PML, PML, PML)
    return ertm.Config(nx=nx, ny=ny, nz=nz, dx=H, dy=H, dz=H, dt_ms=DT_MS, nt=nt, order=8,
                       boundary=ertm.BOUNDARY_CPML, pml=pml, autotune=autotune)
