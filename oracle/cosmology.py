"""astropy's Planck18 background restated (test infrastructure only, see
``oracle/__init__.py``).

The reference converts redshifts with ``astropy.cosmology.Planck18`` when the
config's ``cosmology`` has no ``Omega0`` (src/cosmonpc/catalog_processor.py:
610-625).  astropy (>= 6.1.7, not installed here) defines that realisation as
a flat FLRW model with H0 = 67.66 km/s/Mpc, Om0 = 0.30966, Tcmb0 = 2.7255 K,
Neff = 3.046 and neutrino masses (0, 0, 0.06) eV; its published background
formulas, restated with CODATA 2018 constants:

* Ogamma0 = (4 sigma_SB / c^3) Tcmb0^4 / rho_crit0, rho_crit0 = 3 H0^2 / (8 pi G);
* neutrino density relative to photons (Komatsu et al. 2011, eq. 26 fit), for
  massive neutrinos of y = m c^2 / (k_B T_nu0), T_nu0 = (4/11)^(1/3) Tcmb0:
  n(z) = (7/8)(4/11)^(4/3) (Neff/3) [sum (1 + (0.3173 y/(1+z))^1.83)^(1/1.83) + N_massless];
* E(z)^2 = (1+z)^2 ((Or (1+z) + Om0)(1+z)) + Ode0 with Or = Ogamma0 (1 + n(z)),
  Ode0 = 1 - Om0 - Ogamma0 (1 + n(0));
* comoving distance (c / H0) int_0^z dz'/E(z') (astropy: scipy quad).
"""
from __future__ import annotations

import numpy as np
from scipy.integrate import quad

H0 = 67.66
OM0 = 0.30966
TCMB0 = 2.7255
NEFF = 3.046
M_NU = 0.06
C_KMS = 299792.458


def _constants():
    sigma_sb, c, G = 5.670374419e-8, 299792458.0, 6.67430e-11
    kB_eV = 1.380649e-23 / 1.602176634e-19
    mpc = 3.0856775814913673e22
    h0_si = H0 * 1000.0 / mpc
    rho_crit = 3.0 * h0_si ** 2 / (8.0 * np.pi * G)
    ogamma0 = (4.0 * sigma_sb / c ** 3) * TCMB0 ** 4 / rho_crit
    nu_y = M_NU / (kB_eV * 0.7137658555036082 * TCMB0)
    return ogamma0, nu_y


OGAMMA0, NU_Y = _constants()
NU_PREFAC = 0.22710731766 * (NEFF / 3.0)


def nu_relative_density(z):
    zp1 = 1.0 + np.asarray(z, dtype=np.float64)
    return NU_PREFAC * ((1.0 + (0.3173 * NU_Y / zp1) ** 1.83) ** 0.54644808743 + 2.0)


ODE0 = 1.0 - OM0 - OGAMMA0 - OGAMMA0 * nu_relative_density(0.0)


def efunc(z):
    zp1 = 1.0 + np.asarray(z, dtype=np.float64)
    o_r = OGAMMA0 * (1.0 + nu_relative_density(z))
    return np.sqrt(zp1 ** 2 * ((o_r * zp1 + OM0) * zp1 + 0.0) + ODE0)


def comoving_distance_mpc(z):
    """Comoving distance in Mpc (not Mpc/h) by scipy quad per redshift."""
    zz = np.atleast_1d(np.asarray(z, dtype=np.float64))
    uniq, inv = np.unique(zz, return_inverse=True)
    vals = np.array([quad(lambda t: 1.0 / float(efunc(t)), 0.0, zi, epsabs=0.0, epsrel=1e-13, limit=200)[0]
                     for zi in uniq])
    return (vals[inv] * (C_KMS / H0)).reshape(np.shape(z))
