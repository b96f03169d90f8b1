"""Seeded synthetic earth models and survey geometries.

No public benchmark data ship with the reference (its example model is a
git-LFS pointer and its salt model path is hard-coded to a file that is not
in the repository), so every workload here is generated from a fixed seed:
layered vp with optional Gaussian anomaly or dipping interfaces,
vs = vp / 1.732 and rho = 310 * vp**0.25 (Gardner), positions given as
cell index * spacing in metres, and T = (nt - 0.5) * dt so that
ntime = ceil(T / dt) is unambiguous in float.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Survey:
    """A full problem description in the reference's units.

    Arrays vp/vs/rho are float32 of shape (nz, ny, nx) on gridphy (x fastest
    in memory).  shots/recvs: float32 (n, 3) positions in metres.
    """
    nx: int
    ny: int
    nz: int
    pml: int
    dx: float
    dy: float
    dz: float
    dt: float
    fm: float
    nt: int
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    shots: np.ndarray
    recvs: np.ndarray
    rec_width: int = 1
    name: str = "survey"
    seed: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def T(self) -> float:
        return float(np.float32((self.nt - 0.5) * self.dt))

    @property
    def n_ext(self) -> int:
        return (self.nx + 2 * self.pml) * (self.ny + 2 * self.pml) * (self.nz + 2 * self.pml)

    @property
    def n_phy(self) -> int:
        return self.nx * self.ny * self.nz


def gardner(vp: np.ndarray):
    vp = vp.astype(np.float32)
    vs = (vp / np.float32(1.732)).astype(np.float32)
    rho = (np.float32(310.0) * np.power(vp, np.float32(0.25))).astype(np.float32)
    return vp, vs, rho


def layered_vp(nx, ny, nz, seed, n_layers=3, vmin=2000.0, vmax=4000.0, iface_range=None,
               dip=False, anomaly=None) -> np.ndarray:
    """Layered vp (nz, ny, nx).  Interface depths (in cells) are drawn in
    iface_range (default the middle 80 % of z); with dip=True each interface
    gets a random planar dip of up to ~10 degrees.  anomaly = (amplitude,
    sigma_cells) adds a Gaussian vp perturbation at the grid centre."""
    rng = np.random.default_rng(seed)
    lo, hi = iface_range if iface_range else (0.1 * nz, 0.9 * nz)
    depths = np.sort(rng.uniform(lo, hi, size=n_layers - 1))
    vels = rng.uniform(vmin, vmax, size=n_layers).astype(np.float64)
    z = np.arange(nz, dtype=np.float64)[:, None, None]
    x = np.arange(nx, dtype=np.float64)[None, None, :]
    y = np.arange(ny, dtype=np.float64)[None, :, None]
    vp = np.full((nz, ny, nx), vels[0])
    for li, d in enumerate(depths):
        if dip:
            sx, sy = rng.uniform(-0.18, 0.18, size=2)
            surf = d + sx * (x - nx / 2) + sy * (y - ny / 2)
        else:
            surf = d + 0 * x + 0 * y
        vp = np.where(z >= surf, vels[li + 1], vp)
    if anomaly is not None:
        amp, sig = anomaly
        cz, cy, cx = (nz - 1) / 2, (ny - 1) / 2, (nx - 1) / 2
        g = np.exp(-((z - cz) ** 2 + (y - cy) ** 2 + (x - cx) ** 2) / (2.0 * sig * sig))
        vp = vp * (1.0 + amp * g)
    return vp.astype(np.float32)


def _pos(idx, d):
    a = np.asarray(idx, dtype=np.float64).reshape(-1, 3)
    return (a * np.asarray(d, dtype=np.float64)[None, :]).astype(np.float32)


def small_case(n=(24, 20, 18), pml=6, nt=120, seed=7, rec_width=1, n_layers=3, dx=10.0, dt=1e-3,
               fm=25.0, nrec=None, shot_idx=None, anomaly=None) -> Survey:
    """A small, odd-sized problem for parity tests (seconds on the oracle)."""
    nx, ny, nz = n
    vp = layered_vp(nx, ny, nz, seed, n_layers=n_layers, vmin=2000, vmax=3000, anomaly=anomaly)
    vp, vs, rho = gardner(vp)
    d = (dx, dx, dx)
    if shot_idx is None:
        shot_idx = [(nx // 2, ny // 2, 3)]
    rng = np.random.default_rng(seed + 1)
    if nrec is None:
        rx = np.arange(1, nx - 1, 2)
        rec_idx = [(int(i), ny // 2, 2) for i in rx]
    else:
        rec_idx = [(int(rng.integers(0, nx)), int(rng.integers(0, ny)), int(rng.integers(0, nz))) for _ in range(nrec)]
    return Survey(nx, ny, nz, pml, dx, dx, dx, dt, fm, nt, vp, vs, rho, _pos(shot_idx, d), _pos(rec_idx, d),
                  rec_width=rec_width, name=f"small_{nx}x{ny}x{nz}", seed=seed)


def cfg1(seed: int = 1) -> Survey:
    """Plain forward modelling: 100^3 + 10 CPML, d=5 m, dt=0.4 ms, 1000 steps,
    3 flat layers (interfaces in z 25..75), vp U[2000,4000], 20 Hz Ricker at
    cell (15,15,15), 8 receivers along x at y=z=15."""
    n = 100
    vp = layered_vp(n, n, n, seed, n_layers=3, vmin=2000, vmax=4000, iface_range=(25, 75))
    vp, vs, rho = gardner(vp)
    d = (5.0, 5.0, 5.0)
    rec = [(x, 15, 15) for x in range(15, 86, 10)]
    return Survey(n, n, n, 10, 5.0, 5.0, 5.0, 4e-4, 20.0, 1000, vp, vs, rho, _pos([(15, 15, 15)], d),
                  _pos(rec, d), name="cfg1_forward_100", seed=seed)


def cfg2(rec_width: int = 1, seed: int = 2, nt: int = 2000) -> Survey:
    """Plain single-shot RTM: 200^3 + 20 CPML, d=5 m, dt=0.4 ms, 2000 steps,
    6 layers + Gaussian vp anomaly (+-15 %, sigma 20 cells) at the centre,
    source at cell (100,100,5), 200x200 receivers at z=5."""
    n = 200
    vp = layered_vp(n, n, n, seed, n_layers=6, vmin=2000, vmax=4000, anomaly=(0.15, 20.0))
    vp, vs, rho = gardner(vp)
    d = (5.0, 5.0, 5.0)
    jj, ii = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    rec = np.stack([ii.ravel(), jj.ravel(), np.full(n * n, 5)], axis=1)
    return Survey(n, n, n, 20, 5.0, 5.0, 5.0, 4e-4, 20.0, nt, vp, vs, rho, _pos([(100, 100, 5)], d),
                  _pos(rec, d), rec_width=rec_width, name=f"cfg2_rtm_200_w{rec_width}", seed=seed)


def cfg3(nt: int = 3000, seed: int = 3, rec_step: int = 4) -> Survey:
    """Precision form, large model: 676 x 676 x 210 + 20 CPML, d = 10 m,
    dt = 0.8 ms, vp in [1800, 4500] m/s in 4 layers with 3 dipping
    interfaces.  Choices where the configuration is silent: the source at
    the surface centre, depth 5 cells; receivers every rec_step cells on the
    surface grid at z = 5."""
    nx, ny, nz = 676, 676, 210
    vp = layered_vp(nx, ny, nz, seed, n_layers=4, vmin=1800, vmax=4500, dip=True)
    vp, vs, rho = gardner(vp)
    d = (10.0, 10.0, 10.0)
    jj, ii = np.meshgrid(np.arange(0, ny, rec_step), np.arange(0, nx, rec_step), indexing="ij")
    rec = np.stack([ii.ravel(), jj.ravel(), np.full(ii.size, 5)], axis=1)
    return Survey(nx, ny, nz, 20, 10.0, 10.0, 10.0, 8e-4, 20.0, nt, vp, vs, rho, _pos([(nx // 2, ny // 2, 5)], d),
                  _pos(rec, d), name="cfg3_large_676x676x210", seed=seed)


def cfg3_half(seed: int = 3) -> Survey:
    """cfg3 at half resolution, for the FP64 oracle: the same 6760 x 6760 x
    2100 m model (cfg3's generator on 338 x 338 x 105 cells of 20 m), 10
    CPML cells, dt = 1.6 ms (cfg3's Courant number), 1500 steps (its 2.4 s)
    and a 10 Hz Ricker (its points per wavelength); source at the surface
    centre at depth 3 cells, receivers every 2 cells (40 m, as cfg3's) at z = 3."""
    nx, ny, nz = 338, 338, 105
    vp = layered_vp(nx, ny, nz, seed, n_layers=4, vmin=1800, vmax=4500, dip=True)
    vp, vs, rho = gardner(vp)
    d = (20.0, 20.0, 20.0)
    jj, ii = np.meshgrid(np.arange(0, ny, 2), np.arange(0, nx, 2), indexing="ij")
    rec = np.stack([ii.ravel(), jj.ravel(), np.full(ii.size, 3)], axis=1)
    return Survey(nx, ny, nz, 10, 20.0, 20.0, 20.0, 1.6e-3, 10.0, 1500, vp, vs, rho,
                  _pos([(nx // 2, ny // 2, 3)], d), _pos(rec, d), name="cfg3_half_338x338x105", seed=seed)


def scaled_cfg2(n: int, nt: int, rec_width: int = 1, seed: int = 2, pml: int = 20) -> Survey:
    """cfg2's construction at another size (same spacing, source at the
    centre of the surface at depth 5 cells, full receiver plane at z=5)."""
    vp = layered_vp(n, n, n, seed, n_layers=6, vmin=2000, vmax=4000, anomaly=(0.15, n / 10.0))
    vp, vs, rho = gardner(vp)
    d = (5.0, 5.0, 5.0)
    jj, ii = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    rec = np.stack([ii.ravel(), jj.ravel(), np.full(n * n, min(5, n - 1))], axis=1)
    return Survey(n, n, n, pml, 5.0, 5.0, 5.0, 4e-4, 20.0, nt, vp, vs, rho,
                  _pos([(n // 2, n // 2, min(5, n - 1))], d), _pos(rec, d), rec_width=rec_width,
                  name=f"rtm_{n}_w{rec_width}", seed=seed)


def serving_grid(nx: int, ny: int, nz: int, nt: int, seed: int, rec_step: int = 4, pml: int = 20) -> Survey:
    """One request of the serving mix: a seeded 4-layer model with dipping
    interfaces (vp in [2000, 4000] m/s) on nx x ny x nz cells of 5 m, dt =
    0.4 ms, 20 Hz; the source at a seeded surface position at depth 5
    cells; receivers every rec_step cells on the surface grid at z = 5."""
    vp = layered_vp(nx, ny, nz, seed, n_layers=4, vmin=2000, vmax=4000, dip=True)
    vp, vs, rho = gardner(vp)
    d = (5.0, 5.0, 5.0)
    rng = np.random.default_rng(seed + 7)
    src = [(int(rng.integers(nx // 4, 3 * nx // 4)), int(rng.integers(ny // 4, 3 * ny // 4)), min(5, nz - 1))]
    jj, ii = np.meshgrid(np.arange(0, ny, rec_step), np.arange(0, nx, rec_step), indexing="ij")
    rec = np.stack([ii.ravel(), jj.ravel(), np.full(ii.size, min(5, nz - 1))], axis=1)
    return Survey(nx, ny, nz, pml, 5.0, 5.0, 5.0, 4e-4, 20.0, nt, vp, vs, rho, _pos(src, d), _pos(rec, d),
                  name=f"serve_{nx}x{ny}x{nz}", seed=seed)
