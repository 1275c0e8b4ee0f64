"""Seeded synthetic catalogs with the shapes of the benchmark workloads.

The reference validates against external simulation catalogs that are not
shipped with it; the workloads here use seeded lognormal boxes instead:

* a Gaussian field on a 64^3 grid over the box with
  P(k) = 2e4 (k/0.05)^-1.5 exp(-(k/0.5)^2) (Mpc/h)^3,
* delta_LN = exp(g - sigma^2/2) - 1,
* Poisson counts with mean nbar dV (1 + delta_LN), nbar = Np / L^3,
  positions uniform inside each cell in float64,
* redshift-space displacement along z: z += 0.01 v_z with v_z ~ N(0, 300 km/s)
  (the (1+z)/(100 E(z)) factor of the reference's RSD at a = 1), then wrapped
  into [0, L).  Box ``.npy`` catalogs carry positions with RSD already applied,
  because the reference's ``.npy`` reader ignores velocities
  (``src/cosmonpc/catalog_processor.py:354-386``).
"""
from __future__ import annotations

import numpy as np

BASE_SEED = 20261203


def lognormal_box(n_particles, boxsize, seed, grid=64, rsd_sigma=300.0, pk_amp=2.0e4):
    """Return an (Np, 3) float64 array of positions in [0, boxsize)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = float(boxsize)
    n = int(grid)
    kf = 2.0 * np.pi / L
    kx = np.fft.fftfreq(n, 1.0 / n) * kf
    kz = np.fft.rfftfreq(n, 1.0 / n) * kf
    kk = np.sqrt(kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2)
    with np.errstate(divide="ignore"):
        pk = pk_amp * (kk / 0.05) ** -1.5 * np.exp(-((kk / 0.5) ** 2))
    pk[0, 0, 0] = 0.0
    vol = L ** 3
    amp = np.sqrt(pk * n ** 3 / vol)
    white = rng.standard_normal((n, n, n))
    g = np.fft.irfftn(np.fft.rfftn(white) * amp, s=(n, n, n), axes=(0, 1, 2))
    sigma2 = g.var()
    dln = np.exp(g - 0.5 * sigma2) - 1.0
    nbar = n_particles / vol
    dv = vol / n ** 3
    counts = rng.poisson(nbar * dv * (1.0 + dln)).ravel()
    total = int(counts.sum())
    cell = np.repeat(np.arange(n ** 3, dtype=np.int64), counts)
    ix, rem = np.divmod(cell, n * n)
    iy, iz = np.divmod(rem, n)
    h = L / n
    pos = np.empty((total, 3), dtype=np.float64)
    u = rng.random((total, 3))
    pos[:, 0] = (ix + u[:, 0]) * h
    pos[:, 1] = (iy + u[:, 1]) * h
    pos[:, 2] = (iz + u[:, 2]) * h
    if rsd_sigma:
        vz = rng.normal(0.0, rsd_sigma, total)
        pos[:, 2] = pos[:, 2] + 0.01 * vz
    pos %= L
    return pos


def write_npy_catalog(path, positions, weights=None):
    """Write a box catalog in the reference's ``.npy`` layout (columns x, y, z[, w])."""
    if weights is None:
        arr = np.ascontiguousarray(positions, dtype=np.float64)
    else:
        arr = np.column_stack([positions, weights]).astype(np.float64)
    np.save(path, arr)
    return path
