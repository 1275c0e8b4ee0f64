"""Host-side FP64 angular algebra (scalars and short vectors only).

Restates, without sympy at run time, the small symbolic pieces of the
reference (src/cosmonpc/math_evaluator.py):

* Wigner 3j symbols by the Racah formula in exact integer arithmetic
  (replaces sympy ``wigner_3j(...).evalf()``, math_evaluator.py:312-355).
* Magnetic sub-configurations for box / survey geometry (same enumeration
  order as math_evaluator.py:312-355).
* Spherical-harmonic descriptors for the device kernels: the complex Y_lm of
  math_evaluator.py:35-131 written as norm * Q_l^|m|(z) * (x + i y)^|m| with the
  Condon-Shortley phase inside Q, plus the value the reference's polynomial takes
  at the origin (used only for the k = 0 mode).
* Associated Legendre values with sympy's conventions, the q_l kernel of the
  analytical S3 shot noise and the valid k3-bin mask (math_evaluator.py:389-451,
  :592-616).
"""
from __future__ import annotations

import ctypes
import functools
import math
from fractions import Fraction

import numpy as np


# ------------------------------------------------------------ Wigner 3j
def _fact(n):
    return math.factorial(n)


@functools.lru_cache(maxsize=None)
def wigner3j(j1, j2, j3, m1, m2, m3):
    """Wigner 3j symbol for integer arguments (Racah formula), as float64."""
    if m1 + m2 + m3 != 0:
        return 0.0
    if j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    tri = Fraction(_fact(j1 + j2 - j3) * _fact(j1 - j2 + j3) * _fact(-j1 + j2 + j3), _fact(j1 + j2 + j3 + 1))
    pref = tri * (_fact(j1 + m1) * _fact(j1 - m1) * _fact(j2 + m2) * _fact(j2 - m2)
                  * _fact(j3 + m3) * _fact(j3 - m3))
    kmin = max(0, j2 - j3 - m1, j1 - j3 + m2)
    kmax = min(j1 + j2 - j3, j1 - m1, j2 + m2)
    s = Fraction(0)
    for k in range(kmin, kmax + 1):
        den = (_fact(k) * _fact(j3 - j2 + k + m1) * _fact(j3 - j1 + k - m2)
               * _fact(j1 + j2 - j3 - k) * _fact(j1 - k - m1) * _fact(j2 - k + m2))
        s += Fraction((-1) ** k, den)
    if s == 0:
        return 0.0
    sign = (-1) ** (j1 - j2 - m3) * (1 if s > 0 else -1)
    val2 = pref * s * s
    # sqrt of an exact rational, correctly rounded to double
    num, den = val2.numerator, val2.denominator
    scale = 200
    r = math.isqrt((num << (2 * scale)) // den)
    return float(sign * Fraction(r, 1 << scale))


def magnetic_configs_box(l1, l2, L):
    """(m1, m2, M=0) with m1 >= 0, m1 + m2 = 0 (math_evaluator.py:312-331)."""
    cfgs, vals = [], []
    for m1 in range(0, l1 + 1):
        for m2 in range(-l2, l2 + 1):
            if m1 + m2 == 0:
                cfgs.append((m1, m2, 0))
                vals.append(wigner3j(l1, l2, L, m1, m2, 0))
    return cfgs, vals


def magnetic_configs_survey(l1, l2, L):
    """Half of the (m1, m2, M) set up to and including (0,0,0) (math_evaluator.py:334-355)."""
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


# ----------------------------------------------------- Legendre algebra
@functools.lru_cache(maxsize=None)
def legendre_coeffs(l):
    """Exact coefficients of P_l(x), constant term first (Bonnet recursion)."""
    p0, p1 = [Fraction(1)], [Fraction(0), Fraction(1)]
    if l == 0:
        return tuple(p0)
    for n in range(1, l):
        nxt = [Fraction(0)] * (n + 2)
        for i, c in enumerate(p1):
            nxt[i + 1] += Fraction(2 * n + 1, n + 1) * c
        for i, c in enumerate(p0):
            nxt[i] -= Fraction(n, n + 1) * c
        p0, p1 = p1, nxt
    return tuple(p1)


@functools.lru_cache(maxsize=None)
def reduced_assoc_coeffs(l, m):
    """Coefficients of Q_l^m(z) = (-1)^m d^m P_l / dz^m (m >= 0), constant first."""
    c = list(legendre_coeffs(l))
    for _ in range(m):
        c = [c[i] * i for i in range(1, len(c))] or [Fraction(0)]
    sign = -1 if m % 2 else 1
    return tuple(sign * x for x in c)


def assoc_legendre(l, m, mu):
    """P_l^m(mu) with sympy's conventions (Condon-Shortley phase; m < 0 via
    P_l^{-m} = (-1)^m (l-m)!/(l+m)! P_l^m)."""
    ma = abs(m)
    if ma > l:
        return 0.0
    q = reduced_assoc_coeffs(l, ma)
    poly = 0.0
    for c in reversed(q):
        poly = poly * mu + float(c)
    val = poly * (1.0 - mu * mu) ** (0.5 * ma) if ma else poly
    if m < 0:
        val *= (-1) ** ma * math.factorial(l - ma) / math.factorial(l + ma)
    return val


# ------------------------------------------------------ harmonic tables
class Harmonic(ctypes.Structure):
    """Mirror of ``cnpc_harmonic`` in include/cosmonpc_b200.h."""

    _fields_ = [("l", ctypes.c_int), ("m", ctypes.c_int), ("norm", ctypes.c_double),
                ("coef", ctypes.c_double * 9), ("origin_re", ctypes.c_double),
                ("origin_im", ctypes.c_double)]


def ylm_norm(l, m, racah):
    ma = abs(m)
    n = math.sqrt(math.factorial(l - ma) / math.factorial(l + ma))
    if not racah:
        n *= math.sqrt((2 * l + 1) / (4 * np.pi))
    return n


def ylm_origin_value(l, m, racah):
    """Value of the reference's Y_lm polynomial at (0, 0, 0).

    The reference's sympy construction leaves a constant term only for m = 0
    and l in {0, 4, 6, 8} (the l = 2 numerator collapses to a homogeneous
    quadratic), so the k = 0 mode sees P_l(0) * norm there and 0 elsewhere.
    """
    if m != 0 or l == 2 or l % 2:
        return 0.0
    return float(legendre_coeffs(l)[0]) * ylm_norm(l, 0, racah)


def harmonic(l, m, racah=True):
    if l < 0 or l > 8 or abs(m) > l:
        raise ValueError("harmonic needs 0 <= l <= 8 and |m| <= l")
    h = Harmonic()
    h.l, h.m = l, m
    h.norm = ylm_norm(l, m, racah)
    q = reduced_assoc_coeffs(l, abs(m))
    for i in range(9):
        h.coef[i] = float(q[i]) if i < len(q) else 0.0
    h.origin_re = ylm_origin_value(l, m, racah)
    h.origin_im = 0.0
    return h


def ylm_numpy(l, m, x, y, z, racah=True):
    """Host evaluation of the same harmonic (used for small host-side terms)."""
    h = harmonic(l, m, racah)
    ma = abs(m)
    p = np.zeros_like(np.asarray(z, dtype=np.float64))
    for c in reversed(h.coef[: l - ma + 1]):
        p = p * z + c
    v = h.norm * p * (np.asarray(x) + 1j * np.asarray(y)) ** ma
    if m < 0:
        v = (-1) ** ma * np.conj(v)
    return v


# ------------------------------------------------------ S3 shot noise
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
    """q_{l1 l2 L}(k1, k2, k3) on the k3 bins (math_evaluator.py:592-616)."""
    q = np.zeros(len(k3_eff))
    lmin = min(l1, l2)
    for n in range(-lmin, lmin + 1):
        tj = wigner3j(l1, l2, L, n, -n, 0)
        a13 = _al_eff(l1, n, k_eff[i], k_eff[j], k3_eff, "13")
        a23 = _al_eff(l2, -n, k_eff[i], k_eff[j], k3_eff, "23")
        q += (-1) ** n * tj * a13 * a23
    return q


def valid_k3_bins(k1, k2, k_min, k_max, k_bins):
    """math_evaluator.py:446-450."""
    e = np.linspace(2 * k_min, 2 * k_max, 2 * k_bins + 1)[:-1]
    c = 0.5 * (e[1:] + e[:-1])
    return np.logical_and(c >= abs(k1 - k2), c <= (k1 + k2))


def assoc_legendre_array(l, m, mu):
    """Vectorised ``assoc_legendre`` (same conventions) over an array of mu."""
    ma = abs(m)
    mu = np.asarray(mu, dtype=np.float64)
    if ma > l:
        return np.zeros_like(mu)
    q = reduced_assoc_coeffs(l, ma)
    poly = np.zeros_like(mu)
    for c in reversed(q):
        poly = poly * mu + float(c)
    with np.errstate(invalid="ignore"):
        val = poly * (1.0 - mu * mu) ** (0.5 * ma) if ma else poly
    if m < 0:
        val = val * ((-1) ** ma * math.factorial(l - ma) / math.factorial(l + ma))
    return val


def q_ells_matrix(k1s, l1, l2, L, k3s):
    """q_{l1 l2 L}(k1_i, k1_j, k3_t) for every (i, j, t) at once
    (math_evaluator.py:560-616 evaluated on arrays): shape (B, B, K3)."""
    k1 = np.asarray(k1s, dtype=np.float64)[:, None, None]
    k2 = np.asarray(k1s, dtype=np.float64)[None, :, None]
    k3 = np.asarray(k3s, dtype=np.float64)[None, None, :]
    with np.errstate(invalid="ignore", divide="ignore"):
        valid = np.logical_and(np.abs(k1 - k2) <= k3, k3 <= (k1 + k2))
        mu13 = np.where(valid, (k3 ** 2 + k1 ** 2 - k2 ** 2) / (2 * k1 * k3), 0.0)
        mu23 = np.where(valid, (k3 ** 2 + k2 ** 2 - k1 ** 2) / (2 * k2 * k3), 0.0)
    q = np.zeros(valid.shape)
    lmin = min(l1, l2)
    for n in range(-lmin, lmin + 1):
        tj = wigner3j(l1, l2, L, n, -n, 0)
        if tj == 0.0:
            continue
        a13 = np.where(valid, assoc_legendre_array(l1, n, mu13), 0.0) * (-1) ** (l1 + n)
        a23 = np.where(valid, assoc_legendre_array(l2, -n, mu23), 0.0) * (-1) ** (l2 - n)
        q += (-1) ** n * tj * a13 * a23
    return q


def s3_analytic(total_sum, k_num_k3, k_edge, k3_center, q, diagonal):
    """Analytical S3 contraction (clustering_estimator.py:1081-1180) given the
    q kernel array from ``q_ells_matrix``; returns the (unnormalised) S3."""
    k_bins = len(k_edge) - 1
    weighted = k_num_k3 / k3_center
    terms = total_sum / k3_center
    if diagonal:
        s3 = np.zeros(k_bins, dtype="complex128")
        for i in range(k_bins):
            numer = np.sum(q[i, i] * terms)
            denom = np.sum(weighted[: 2 * i + 1])
            if denom > 0:
                s3[i] = numer / denom
        return s3
    k_center = 0.5 * (k_edge[1:] + k_edge[:-1])
    kc1 = k_center[:, None, None]
    kc2 = k_center[None, :, None]
    k3c = k3_center[None, None, :]
    vb = np.logical_and(k3c >= np.abs(kc1 - kc2), k3c <= (kc1 + kc2))
    numer = np.sum(q * terms[None, None, :], axis=2)
    denom = np.sum(weighted[None, None, :] * vb, axis=2)
    s3 = np.zeros((k_bins, k_bins), dtype="complex128")
    ok = denom > 0
    s3[ok] = numer[ok] / denom[ok]
    return s3
