"""Angular algebra of CosmoNPC restated for the oracle (sympy + numpy, FP64).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

* ``ylm_function`` follows ``src/cosmonpc/math_evaluator.py:35-131``: the complex
  spherical harmonic built as a sympy polynomial in (xhat, yhat, zhat) with the
  Condon-Shortley phase, optional Racah factor sqrt(4 pi / (2l+1)), conjugation
  rule for m < 0, then evaluated with numpy.  The steps are kept alike because the
  polynomial form (not only its values on the unit sphere) decides the value at
  the k = 0 mode, where the reference evaluates it at (0, 0, 0).
* ``legendre_function`` follows ``math_evaluator.py:134-197``.
* ``wigner3j`` / ``magnetic_configs_box`` / ``magnetic_configs_survey`` follow
  ``math_evaluator.py:312-355`` (sympy's wigner_3j).
* ``q_ells_eff`` / ``valid_k3_bins`` follow ``math_evaluator.py:418-451`` and
  ``math_evaluator.py:592-616``; associated Legendre values come from sympy's
  ``assoc_legendre`` polynomial evaluated by numpy.
"""
from __future__ import annotations

import functools

import numpy as np
import sympy as sp


@functools.lru_cache(maxsize=None)
def _ylm_expr(l, m, racah):
    x, y, z = sp.symbols("x y z", real=True)
    r = sp.symbols("r", real=True, positive=True)
    xh, yh, zh = sp.symbols("xhat yhat zhat", real=True)
    phi, theta = sp.symbols("phi theta")
    defs = [
        (sp.sin(phi), y / sp.sqrt(x ** 2 + y ** 2)),
        (sp.cos(phi), x / sp.sqrt(x ** 2 + y ** 2)),
        (sp.cos(theta), z / sp.sqrt(x ** 2 + y ** 2 + z ** 2)),
    ]
    amp = sp.sqrt((2 * l + 1) / (4 * np.pi) * sp.factorial(l - abs(m)) / sp.factorial(l + abs(m)))
    e = sp.assoc_legendre(l, abs(m), sp.cos(theta)) * (sp.cos(phi) + sp.I * sp.sin(phi)) ** abs(m)
    e = e.subs(defs)
    e = sp.together(e).subs(x ** 2 + y ** 2 + z ** 2, r ** 2)
    e = amp * e.expand().subs([(x / r, xh), (y / r, yh), (z / r, zh)])
    if racah:
        e = e * sp.sqrt(4 * np.pi / (2 * l + 1))
    if m < 0:
        e = (-1) ** m * sp.conjugate(e)
    e = sp.simplify(e)
    return e, (xh, yh, zh)


@functools.lru_cache(maxsize=None)
def ylm_function(l, m, racah=False):
    """Return f(xhat, yhat, zhat) -> complex Y_lm (numpy arrays in, complex128 out)."""
    if abs(m) > l:
        raise ValueError("abs(m) must be <= l")
    e, syms = _ylm_expr(l, m, racah)
    f = sp.lambdify(syms, e, "numpy")

    def ylm(xh, yh, zh):
        out = f(xh, yh, zh)
        return np.broadcast_to(np.asarray(out, dtype=np.complex128),
                               np.broadcast(xh, yh, zh).shape)

    ylm.expr = e
    return ylm


@functools.lru_cache(maxsize=None)
def legendre_function(ell, rx, ry, rz):
    if not np.isclose(rx * rx + ry * ry + rz * rz, 1.0):
        raise ValueError("(r_xhat, r_yhat, r_zhat) must form a unit vector")
    kx, ky, kz = sp.symbols("k_xhat k_yhat k_zhat", real=True)
    c = sp.Symbol("cos_theta", real=True)
    e = sp.simplify(sp.legendre(ell, c).subs(c, rx * kx + ry * ky + rz * kz))
    f = sp.lambdify((kx, ky, kz), e, "numpy")

    def pl(a, b, d):
        return np.broadcast_to(np.asarray(f(a, b, d), dtype=np.float64),
                               np.broadcast(a, b, d).shape)

    return pl


@functools.lru_cache(maxsize=None)
def wigner3j(j1, j2, j3, m1, m2, m3):
    from sympy.physics.wigner import wigner_3j

    return np.float64(wigner_3j(j1, j2, j3, m1, m2, m3).evalf())


def magnetic_configs_box(l1, l2, L):
    cfgs, vals = [], []
    for m1 in range(0, l1 + 1):
        for m2 in range(-l2, l2 + 1):
            if m1 + m2 == 0:
                cfgs.append((m1, m2, 0))
                vals.append(wigner3j(l1, l2, L, m1, m2, 0))
    return cfgs, vals


def magnetic_configs_survey(l1, l2, L):
    cfgs, vals = [], []
    for M in range(-L, L + 1):
        for m1 in range(-l1, l1 + 1):
            m2 = -M - m1
            if -l2 <= m2 <= l2:
                cfgs.append((m1, m2, M))
                vals.append(wigner3j(l1, l2, L, m1, m2, M))
                if (m1, m2, M) == (0, 0, 0):
                    return cfgs, vals
    return cfgs, vals


@functools.lru_cache(maxsize=None)
def _assoc_legendre_fn(l, m):
    mu = sp.Symbol("mu", real=True)
    return sp.lambdify(mu, sp.assoc_legendre(l, m, mu), "numpy")


def assoc_legendre(l, m, mu):
    return np.float64(_assoc_legendre_fn(l, m)(np.float64(mu)))


def _al_eff(l, m, k1, k2, k3_eff, mode):
    out = np.zeros(len(k3_eff))
    for i, k3 in enumerate(k3_eff):
        if abs(k1 - k2) <= k3 <= (k1 + k2):
            if mode == "13":
                mu = (k3 ** 2 + k1 ** 2 - k2 ** 2) / (2 * k1 * k3)
            else:
                mu = (k3 ** 2 + k2 ** 2 - k1 ** 2) / (2 * k2 * k3)
            out[i] = assoc_legendre(l, m, mu)
    out *= (-1) ** (l + m)
    return out


def q_ells_eff(i, j, k_eff, l1, l2, L, k3_eff):
    q = np.zeros(len(k3_eff))
    lmin = min(l1, l2)
    for n in range(-lmin, lmin + 1):
        tj = wigner3j(l1, l2, L, n, -n, 0)
        a13 = _al_eff(l1, n, k_eff[i], k_eff[j], k3_eff, "13")
        a23 = _al_eff(l2, -n, k_eff[i], k_eff[j], k3_eff, "23")
        q += (-1) ** n * tj * a13 * a23
    return q


def valid_k3_bins(k1, k2, k_min, k_max, k_bins):
    e = np.linspace(2 * k_min, 2 * k_max, 2 * k_bins + 1)[:-1]
    c = 0.5 * (e[1:] + e[:-1])
    return np.logical_and(c >= abs(k1 - k2), c <= (k1 + k2))
