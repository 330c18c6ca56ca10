"""Seeded synthetic workloads: cubic-perovskite ABO3 supercells and raster scans.

No public dataset is involved; the benchmark configurations define their own
generator and this module fixes its free choices:

* lattice a = 3.905 Angstrom; A at (0,0,0), B at (1/2,1/2,1/2), O at (1/2,1/2,0),
  (1/2,0,1/2), (0,1/2,1/2); slices of c/2 = 1.95 Angstrom hold alternately the AO
  plane (A at (0,0), O at (1/2,1/2)) and the BO2 plane (B at (1/2,1/2), O at
  (1/2,0) and (0,1/2));
* the pixel pitch makes the supercell exactly periodic: calib = cells * a / N
  (0.244063 Angstrom for 8/128, 16/256 and 32/512);
* every atom gets its own seeded in-plane Gaussian displacement (sigma 0.05 A,
  ``numpy.random.default_rng(seed)``);
* an atom's projected potential is Z**0.7 * (12 exp(-r^2 / (2 * 0.15^2)) +
  4 exp(-r^2 / (2 * 0.45^2))) volt-Angstrom (A-site Z=38, B-site Z=22, O Z=8),
  summed periodically over a 4-sigma window of the wider Gaussian;
* scans are raster grids centred on the probe, with positions in Angstrom handed
  to ``DetectorConfig.scan_positions_px`` (the reference's ``stem_4d`` applies
  that field as an Angstrom shift).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

LATTICE_A = 3.905
SLICE_DZ = 1.95
Z_A, Z_B, Z_O = 38, 22, 8
GAUSS_AMP = (12.0, 4.0)
GAUSS_SIGMA = (0.15, 0.45)


@dataclass(frozen=True)
class Workload:
    """One benchmark configuration."""

    name: str
    n: int
    cells: int
    num_slices: int
    scan: tuple
    voltage_kv: float
    aperture_mrad: float
    defocus_ang: float = 0.0
    c3_ang: float = 0.0
    phonon_configs: int = 1
    seed: int = 0

    @property
    def calib(self) -> float:
        return self.cells * LATTICE_A / self.n

    @property
    def num_probes(self) -> int:
        return int(self.scan[0] * self.scan[1])


# The benchmark configurations: plain 128^2 (CPU-runnable), batched 256^2
# (headline), large-grid 512^2 with four frozen-phonon configurations.
CONFIG1 = Workload("perovskite-8x8-128px-20sl-16x16scan", 128, 8, 20, (16, 16), 300.0, 20.0, seed=1)
# Cs = 1 um is c3_ang = 1e-3: the reference scales C3 by 1e7 (simulations.py:491-497)
CONFIG2 = Workload("perovskite-16x16-256px-50sl-64x64scan", 256, 16, 50, (64, 64), 200.0, 25.0,
                   defocus_ang=-50.0, c3_ang=1e-3, seed=2)
CONFIG3 = Workload("perovskite-32x32-512px-100sl-128x128scan", 512, 32, 100, (128, 128), 300.0, 30.0,
                   phonon_configs=4, seed=3)


def _plane_sites(cells: int, odd: bool) -> tuple:
    """Fractional in-plane sites and Z of one slice."""
    i, j = np.meshgrid(np.arange(cells), np.arange(cells), indexing="ij")
    i = i.ravel().astype(np.float64)
    j = j.ravel().astype(np.float64)
    if not odd:  # AO plane
        ys = [i, i + 0.5]
        xs = [j, j + 0.5]
        zs = [Z_A, Z_O]
    else:  # BO2 plane
        ys = [i + 0.5, i + 0.5, i]
        xs = [j + 0.5, j, j + 0.5]
        zs = [Z_B, Z_O, Z_O]
    y = np.concatenate(ys)
    x = np.concatenate(xs)
    z = np.concatenate([np.full(i.size, zz, np.float64) for zz in zs])
    return y, x, z


def slice_potential(n: int, cells: int, slice_index: int, rng: np.random.Generator,
                    sigma_disp: float = 0.05) -> np.ndarray:
    """Projected potential (n, n) of one slice in volt-Angstrom."""
    calib = cells * LATTICE_A / n
    y, x, z = _plane_sites(cells, slice_index % 2 == 1)
    disp = rng.normal(0.0, sigma_disp, size=(2, y.size))
    py = (y * LATTICE_A + disp[0]) / calib  # pixel coordinates
    px = (x * LATTICE_A + disp[1]) / calib
    half = int(np.ceil(4 * GAUSS_SIGMA[1] / calib))
    off = np.arange(-half, half + 1)
    cy = np.floor(py).astype(np.int64)
    cx = np.floor(px).astype(np.int64)
    gy = cy[:, None, None] + off[None, :, None]
    gx = cx[:, None, None] + off[None, None, :]
    dy = (gy - py[:, None, None]) * calib
    dx = (gx - px[:, None, None]) * calib
    r2 = dy * dy + dx * dx
    amp = np.power(z, 0.7)[:, None, None]
    val = amp * (GAUSS_AMP[0] * np.exp(-r2 / (2 * GAUSS_SIGMA[0] ** 2)) +
                 GAUSS_AMP[1] * np.exp(-r2 / (2 * GAUSS_SIGMA[1] ** 2)))
    idx = (np.mod(gy, n) * n + np.mod(gx, n)).ravel()
    out = np.bincount(idx, weights=val.ravel(), minlength=n * n)
    return out.reshape(n, n)


def potential_slices(w: Workload, phonon: int = 0, num_slices: Optional[int] = None) -> np.ndarray:
    """Slices (N, N, S) float32 for frozen-phonon configuration ``phonon``."""
    s_total = w.num_slices if num_slices is None else num_slices
    rng = np.random.default_rng([w.seed, phonon])
    out = np.empty((w.n, w.n, s_total), np.float32)
    for s in range(s_total):
        out[:, :, s] = slice_potential(w.n, w.cells, s, rng)
    return out


def raster_positions(w: Workload, scan=None) -> np.ndarray:
    """Raster scan (P, 2) of (y, x) shifts in Angstrom spanning the field of view."""
    ny, nx = w.scan if scan is None else scan
    fov = w.n * w.calib
    ys = (np.arange(ny) - (ny - 1) / 2.0) * (fov / ny)
    xs = (np.arange(nx) - (nx - 1) / 2.0) * (fov / nx)
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    return np.stack([yy.ravel(), xx.ravel()], axis=1)


def algorithmic_flops_per_update(n: int) -> float:
    """Two complex 2-D FFTs (5 N^2 log2 N^2 each) and two complex multiplies (6 N^2)."""
    return 20.0 * n * n * np.log2(n) + 12.0 * n * n


@dataclass(frozen=True)
class GradWorkload:
    """Ptychographic gradient configuration: n x n probe windows over an F x F field."""

    name: str
    n: int
    field_n: int
    cells: int
    num_slices: int
    scan: tuple
    step_px: int
    voltage_kv: float
    aperture_mrad: float
    defocus_ang: float
    c3_ang: float
    dose: float
    seed: int

    @property
    def calib(self) -> float:
        return self.cells * LATTICE_A / self.field_n

    @property
    def num_probes(self) -> int:
        return int(self.scan[0] * self.scan[1])

    def windows(self) -> np.ndarray:
        """(P, 2) int32 window origins: a raster with step_px that keeps windows inside the field."""
        iy, ix = np.meshgrid(np.arange(self.scan[0]), np.arange(self.scan[1]), indexing="ij")
        return np.stack([iy.ravel() * self.step_px, ix.ravel() * self.step_px], axis=1).astype(np.int32)

    def field(self, phonon: int = 0) -> np.ndarray:
        w = Workload(self.name, self.field_n, self.cells, self.num_slices, self.scan, self.voltage_kv,
                     self.aperture_mrad, seed=self.seed)
        return potential_slices(w, phonon)


# 256^2 windows over a 512^2 field (32x32 cells), 10 slices, 32x32 scan with an 8 px step,
# targets Poisson-noised at 1e4 electrons per pattern.
CONFIG4 = GradWorkload("ptycho-512px-field-256px-window-10sl-32x32scan", 256, 512, 32, 10, (32, 32), 8,
                       200.0, 25.0, -50.0, 1e-3, 1e4, seed=4)


def poisson_targets(patterns: np.ndarray, dose: float, rng: np.random.Generator) -> np.ndarray:
    """Patterns (P, n, n) with Poisson counting noise at ``dose`` electrons per pattern,
    scaled back to the patterns' units."""
    total = patterns.sum(axis=(1, 2), keepdims=True)
    lam = np.clip(patterns, 0, None) / total * dose
    return rng.poisson(lam).astype(np.float64) * total / dose
