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


def lognormal_box(n_particles, boxsize, seed, grid=64, rsd_sigma=300.0, pk_amp=2.0e4,
                  return_field=False):
    """Return an (Np, 3) float64 array of positions in [0, boxsize).

    With ``return_field`` the (grid^3) array 1 + delta_LN is returned instead.
    """
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
    if return_field:
        return 1.0 + dln
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


# ------------------------------------------------------------------ survey
# Survey-like catalogs in the reference's FITS layout (RA, DEC in degrees, Z,
# NZ, WEIGHT_FKP[, WEIGHT_SYSTOT, WEIGHT_NOZ, WEIGHT_CP]).  Angles are uniform
# on the sphere inside an RA/DEC rectangle, redshifts Gaussian and clipped;
# data points are thinned from the same distribution with probability
# proportional to 1 + delta_LN of a lognormal field over the survey's bounding
# box, so the data cluster while the randoms trace the selection function.
# NZ is the data's n(z) histogram divided by the shell volume, the FKP weight
# 1/(1 + P0 NZ).

def _comoving_table(h, omega_m, zmax, n=4096):
    z = np.linspace(0.0, zmax, n)
    inv = 1.0 / np.sqrt(omega_m * (1 + z) ** 3 + (1 - omega_m))
    chi = np.concatenate([[0.0], np.cumsum(0.5 * (inv[1:] + inv[:-1]) * np.diff(z))])
    return z, chi * 299792.458 / 100.0  # Mpc/h


def _sky_sample(rng, n, ra, dec, z_mu, z_sigma, z_clip):
    r = np.deg2rad(rng.uniform(ra[0], ra[1], n))
    s0, s1 = np.sin(np.deg2rad(dec[0])), np.sin(np.deg2rad(dec[1]))
    d = np.arcsin(rng.uniform(s0, s1, n))
    z = np.clip(rng.normal(z_mu, z_sigma, n), z_clip[0], z_clip[1])
    return r, d, z


def lognormal_box_exact(n_particles, boxsize, seed, **kw):
    """:func:`lognormal_box` with exactly ``n_particles`` positions (a random
    subset of a slightly larger draw), as for fixed-size mock catalogs."""
    rng = np.random.Generator(np.random.PCG64(seed + 7919))
    pos = lognormal_box(int(n_particles * 1.02) + 64, boxsize, seed, **kw)
    if len(pos) >= n_particles:
        return pos[np.sort(rng.choice(len(pos), n_particles, replace=False))]
    extra = pos[rng.integers(0, len(pos), n_particles - len(pos))]
    return np.concatenate([pos, extra])


def survey_catalogs(n_data, n_randoms, seed, ra=(150.0, 180.0), dec=(10.0, 35.0), z_mu=0.5,
                    z_sigma=0.05, z_clip=(0.4, 0.6), h=0.6766, omega_m=0.31, p0=1.0e4,
                    boss_weights=False, grid=32, pk_amp=2.0e4):
    """Return (data, randoms) as dicts of float64 columns for :func:`write_fits_catalog`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    zt, ct = _comoving_table(h, omega_m, z_clip[1] * 1.01 + 0.01)

    def xyz(r, d, z):
        chi = np.interp(z, zt, ct)
        return np.column_stack([chi * np.cos(d) * np.cos(r), chi * np.cos(d) * np.sin(r), chi * np.sin(d)])

    rr, rd, rz = _sky_sample(rng, n_randoms, ra, dec, z_mu, z_sigma, z_clip)
    rpos = xyz(rr, rd, rz)
    lo, hi = rpos.min(0), rpos.max(0)
    span = float((hi - lo).max()) * 1.05 + 1e-9
    field = lognormal_box(0, span, int(rng.integers(1 << 31)), grid=grid, rsd_sigma=0.0,
                          pk_amp=pk_amp, return_field=True)
    accept = field / field.max()
    dr, dd, dz = [], [], []
    need = n_data
    while need > 0:
        m = max(4 * need, 1024)
        cr, cd, cz = _sky_sample(rng, m, ra, dec, z_mu, z_sigma, z_clip)
        idx = np.floor((xyz(cr, cd, cz) - lo) / span * grid).astype(np.int64).clip(0, grid - 1)
        keep = rng.random(m) < accept[idx[:, 0], idx[:, 1], idx[:, 2]]
        take = np.flatnonzero(keep)[:need]
        dr.append(cr[take])
        dd.append(cd[take])
        dz.append(cz[take])
        need -= take.size
    dr, dd, dz = np.concatenate(dr), np.concatenate(dd), np.concatenate(dz)
    area = np.deg2rad(ra[1] - ra[0]) * (np.sin(np.deg2rad(dec[1])) - np.sin(np.deg2rad(dec[0])))
    zedges = np.linspace(z_clip[0], z_clip[1], 41)
    shell = area / 3.0 * np.diff(np.interp(zedges, zt, ct) ** 3)
    nz_bin = np.histogram(dz, bins=zedges)[0] / shell

    def cols(r, d, z, data):
        nz = nz_bin[np.clip(np.searchsorted(zedges, z, side="right") - 1, 0, len(shell) - 1)]
        out = {"RA": np.rad2deg(r), "DEC": np.rad2deg(d), "Z": z, "NZ": nz,
               "WEIGHT_FKP": 1.0 / (1.0 + p0 * nz)}
        if boss_weights and data:
            k = len(z)
            out["WEIGHT_SYSTOT"] = rng.uniform(0.9, 1.1, k)
            out["WEIGHT_NOZ"] = 1.0 + (rng.random(k) < 0.05)
            out["WEIGHT_CP"] = 1.0 + (rng.random(k) < 0.05)
        return out

    return cols(dr, dd, dz, True), cols(rr, rd, rz, False)


def write_fits_catalog(path, columns):
    """Write a survey catalog (dict of equal-length columns) as a FITS binary table."""
    from .fits import write_table

    write_table(path, {k: np.asarray(v, dtype=np.float64) for k, v in columns.items()})
    return path
