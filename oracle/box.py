"""CPU restatement (numpy, complex128 full-spectrum fields) of CosmoNPC's box path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every function cites the
reference lines it restates; the arithmetic is FP64/complex128 with full
complex-to-complex transforms, exactly the representation the reference uses
through pmesh (``src/cosmonpc/mesh_generator.py:189-191``).

Reference files: ``mg`` = src/cosmonpc/mesh_generator.py,
``me`` = src/cosmonpc/math_evaluator.py, ``ce`` = src/cosmonpc/clustering_estimator.py.
"""
from __future__ import annotations

import numpy as np

from . import angular
from .pmesh_lite import ParticleMesh, _fftn, _ifftn, paint_mass

ORDER = {"ngp": 1, "cic": 2, "tsc": 3, "pcs": 4}


# ----------------------------------------------------------------- painting
def paint_field(pos, weight, nmesh, boxsize, sampler, interlaced):
    """``pm_painter`` (mg:172-224): mass mesh, interlaced pair combined in k-space.

    Returns the complex128 "real" field exactly as the reference holds it.
    """
    n = int(nmesh)
    L = float(boxsize)
    pm = ParticleMesh([L] * 3, [n] * 3, resampler="nearest" if sampler == "ngp" else sampler)
    order = ORDER[sampler]
    g = np.asarray(pos, dtype=np.float64) * pm.affine.scale
    m1 = paint_mass(g, weight, pm.Nmesh, order)
    if not interlaced:
        return m1.astype(np.complex128)
    m2 = paint_mass(g + 0.5, weight, pm.Nmesh, order)
    N3 = float(n) ** 3
    c1 = _fftn(m1.astype(np.complex128)) / N3
    c2 = _fftn(m2.astype(np.complex128)) / N3
    H = L / n
    kH = 0
    for d in range(3):
        kH = kH + pm.k[d] * H
    c = c1 * 0.5 + c2 * 0.5 * np.exp(0.5 * 1j * kH)
    return _ifftn(c) * N3


# ------------------------------------------------------------ compensation
def _sinc_half(w):
    return np.sinc(0.5 * w / np.pi)


def compensation_kernel(kind, sampler, w):
    """Multiplicative k-space kernel of the window compensation.

    kind = "sinc" (me:206-248, used for interlaced pk and all bk signal terms),
    "shotnoise" (Jing form, me:251-275, non-interlaced pk) or "bknoise"
    (me:278-309, the Sugiyama shot-noise kernel applied to a constant field).
    Returned as the factor v_out / v_in, built per axis in the same order.
    """
    p = ORDER[sampler]
    out = np.ones(np.broadcast(*w).shape)
    for d in range(3):
        wd = w[d]
        if kind == "sinc":
            if p == 1:
                t = _sinc_half(wd)
                t = np.where(wd == 0.0, 1.0, t)
            elif p == 2:
                t = _sinc_half(wd) ** 2
                t = np.where(wd == 0.0, 1.0, t)
            else:
                t = _sinc_half(wd) ** p
            out = out / t
        elif kind == "shotnoise":
            if p == 1:
                continue
            s = np.sin(0.5 * wd) ** 2
            if p == 2:
                c = 1 - 2.0 / 3 * s
            elif p == 3:
                c = 1 - s + 2.0 / 15 * s ** 2
            else:
                c = 1 - 4.0 / 3.0 * s + 2.0 / 5.0 * s ** 2 - 4.0 / 315.0 * s ** 3
            out = out / c ** 0.5
        elif kind == "bknoise":
            if p == 1:
                continue
            s = np.sin(0.5 * wd) ** 2
            t = _sinc_half(wd) ** p
            t = np.where(wd == 0.0, 1.0, t)
            if p == 2:
                c = 1 - 2.0 / 3 * s
            elif p == 3:
                c = 1 - s + 2.0 / 15 * s ** 2
            else:
                c = 1 - 4.0 / 3.0 * s + 2.0 / 5.0 * s ** 2 - 4.0 / 315.0 * s ** 3
            out = out * c / t ** 2
        else:
            raise ValueError(kind)
    return out


# --------------------------------------------------------------- k geometry
class KGeom:
    """k vectors, |k|, unit vectors (me:12-22) and the circular coordinates."""

    def __init__(self, nmesh, boxsize):
        pm = ParticleMesh([boxsize] * 3, [nmesh] * 3)
        self.pm = pm
        self.k = pm.k
        self.w = pm.w
        knorm = np.sqrt(sum(np.real(kk) ** 2 for kk in pm.k))
        self.knorm = knorm
        with np.errstate(invalid="ignore", divide="ignore"):
            self.khat = [np.broadcast_to(kk, knorm.shape) / knorm for kk in pm.k]
        for kh in self.khat:
            kh[0, 0, 0] = 0.0


def kbin_count(k_bins, edges, knorm):
    """``get_kbin_count`` (me:452-481)."""
    kn = knorm.ravel()
    valid = np.logical_and(kn >= edges[0], kn < edges[-1])
    kn = kn[valid]
    idx = np.searchsorted(edges, kn, side="right") - 1
    return (np.bincount(idx, minlength=k_bins).astype("f8"),
            np.bincount(idx, weights=kn, minlength=k_bins).astype("f8"))


def radial_bin(field, k_bins, edges, knorm):
    """``radial_binning`` (me:504-539)."""
    f = np.ascontiguousarray(field).ravel()
    kn = knorm.ravel()
    valid = np.logical_and(kn >= edges[0], kn < edges[-1])
    kn = kn[valid]
    f = f[valid]
    idx = np.searchsorted(edges, kn, side="right") - 1
    if np.iscomplexobj(f):
        s = (np.bincount(idx, weights=np.real(f), minlength=k_bins)
             + 1j * np.bincount(idx, weights=np.imag(f), minlength=k_bins))
        return s.astype(f.dtype, copy=False)
    return np.bincount(idx, weights=f, minlength=k_bins).astype(f.dtype, copy=False)


def _fwd(field):
    N3 = float(field.size)
    return _fftn(np.asarray(field, dtype=np.complex128)) / N3


def _inv(cfield):
    N3 = float(cfield.size)
    return _ifftn(cfield) * N3


# ------------------------------------------------------------------ pk box
def pk_box(field_a, field_b, correlation_mode, nmesh, boxsize, k_min, k_max, k_bins,
           poles, sampler, interlaced, rsd, NZ_a, NZ_b=None):
    """``calculate_power_spectrum_box`` (ce:566-746); returns the result dict."""
    geo = KGeom(nmesh, boxsize)
    edges = np.linspace(k_min, k_max, k_bins + 1)
    kind = "sinc" if interlaced else "shotnoise"
    comp = compensation_kernel(kind, sampler, geo.w)
    ca = _fwd(field_a) * comp
    cb = _fwd(field_b) * comp if correlation_mode == "cross" else ca
    if geo.knorm[0, 0, 0] == 0.0:
        ca[0, 0, 0] = 0.0
    P = np.real(ca) * np.real(cb) + np.imag(ca) * np.imag(cb)
    k_num, ksum = kbin_count(k_bins, edges, geo.knorm)
    res = {"k_eff": ksum / k_num, "k_num": k_num}
    V = float(boxsize) ** 3
    N6 = float(nmesh) ** 6
    P_shot = 1.0 / NZ_a if correlation_mode == "auto" else 0.0
    rsd = np.asarray(rsd, dtype=np.float64)
    for pole in poles:
        if pole & 1:
            r = np.zeros(k_bins).astype("float128")
        else:
            if pole == 0:
                s = radial_bin(P, k_bins, edges, geo.knorm)
            else:
                Lf = angular.legendre_function(pole, float(rsd[0]), float(rsd[1]), float(rsd[2]))
                s = radial_bin(P * Lf(*geo.khat), k_bins, edges, geo.knorm)
            r = s / k_num
            if correlation_mode == "auto":
                r = r * (V ** -1 * N6 / NZ_a ** 2)
            else:
                r = r * (V ** -1 * N6 / (NZ_a * NZ_b))
            if pole == 0:
                r = r - P_shot
            else:
                r = r * (2 * pole + 1)
        res["P%d" % pole] = r
        res["P_shot"] = P_shot
    return res


# ------------------------------------------------------------- bk_sugi box
def bk_sugi_box(field_a, field_b, field_c, correlation_mode, tracer_type, nmesh, boxsize,
                k_min, k_max, k_bins, angu_config, sampler, data_vector_mode,
                shotnoise_mode, N_gal, NZ, return_parts=False, bins=None):
    """``calculate_bk_sugi_box`` (ce:749-1555).

    ``N_gal`` / ``NZ`` are dicts keyed by tracer letter.  The shell fields are
    built without blocking: ``block_size`` only decides which fields are held at
    once in the reference (ce:911-981) and does not change the sums.

    ``bins`` (full mode only): evaluate the triple sums of the signal and of the
    FFT S3 term only for (k1, k2) pairs with both bins in this list; the other
    entries of those matrices are NaN.  Every entry that is computed equals the
    unrestricted run's (the sums of one pair do not depend on other bins), so a
    large mesh can be checked on a fixed subset of its data vector.
    """
    l1, l2, L = angu_config
    n = int(nmesh)
    V = float(boxsize) ** 3
    N3 = float(n) ** 3
    dV = V / N3
    geo = KGeom(n, boxsize)
    edges = np.linspace(k_min, k_max, k_bins + 1)
    N_ells = (2 * l1 + 1) * (2 * l2 + 1) * (2 * L + 1)
    H_ells = angular.wigner3j(l1, l2, L, 0, 0, 0)
    cfgs, tj = angular.magnetic_configs_box(l1, l2, L)
    comp = compensation_kernel("sinc", sampler, geo.w)

    # ce:808-837: delta = rho/dV - NZ, r2c, compensate
    ca = _fwd(np.asarray(field_a) / dV - NZ["a"]) * comp
    cb = cc = None
    if correlation_mode == "cross":
        cb = _fwd(np.asarray(field_b) / dV - NZ["b"]) * comp
        if tracer_type == "abc":
            cc = _fwd(np.asarray(field_c) / dV - NZ["c"]) * comp
    # ce:844-851
    if correlation_mode == "auto":
        G = np.real(_inv(ca))
    else:
        G = np.real(_inv(cc if tracer_type == "abc" else cb))
    k_num, ksum = kbin_count(k_bins, edges, geo.knorm)
    k_eff = ksum / k_num
    masks = [np.logical_and(geo.knorm >= edges[i], geo.knorm < edges[i + 1]) for i in range(k_bins)]
    khat = geo.khat
    same_tracer = correlation_mode == "auto" or tracer_type == "aab"
    leg2_src = ca if tracer_type in ("aaa", "aab") else cb

    sel = list(range(k_bins)) if bins is None else sorted(set(int(b) for b in bins))
    if data_vector_mode == "full":
        total = np.zeros((k_bins, k_bins), dtype=np.complex128)
        for ss, (m1, m2, _) in enumerate(cfgs):
            y1 = angular.ylm_function(l1, m1, True)(*khat)
            y2 = angular.ylm_function(l2, m2, True)(*khat)
            w1 = ca * y1
            w2 = leg2_src * y2
            eq = same_tracer and l1 == l2 and m1 == m2
            cj = same_tracer and l1 == l2 and m1 == -m2
            F1 = {i: _inv(w1 * masks[i]) for i in sel}
            sub = np.full((k_bins, k_bins), np.nan, dtype=np.complex128)
            if eq or cj:
                for i in sel:
                    for j in sel:
                        if j < i:
                            continue
                        F2 = F1[j] if eq else (-1) ** (m1 + l1) * np.conj(F1[j])
                        sub[i, j] = tj[ss] * np.sum(G * F1[i] * F2)
                for i in sel:
                    for j in sel:
                        if j > i:
                            sub[j, i] = sub[i, j] if eq else np.conj(sub[i, j])
            else:
                F2 = {j: _inv(w2 * masks[j]) for j in sel}
                for i in sel:
                    for j in sel:
                        sub[i, j] = tj[ss] * np.sum(G * F1[i] * F2[j])
            del F1
            total += sub if (m1, m2) == (0, 0) else 2 * np.real(sub)
    else:
        total = np.zeros(k_bins, dtype=np.complex128)
        for ss, (m1, m2, _) in enumerate(cfgs):
            y1 = angular.ylm_function(l1, m1, True)(*khat)
            w1 = ca * y1
            w2 = None
            if tracer_type in ("aaa", "aab"):
                if l1 != l2 or m1 != m2:
                    w2 = ca * angular.ylm_function(l2, m2, True)(*khat)
            else:
                w2 = cb * angular.ylm_function(l2, m2, True)(*khat)
            sub = np.zeros(k_bins, dtype=np.complex128)
            for i in range(k_bins):
                F1 = _inv(w1 * masks[i])
                if tracer_type in ("aaa", "aab") and l1 == l2:
                    F2 = F1 if m1 == 0 else (-1) ** (m1 + l1) * np.conj(F1)
                else:
                    F2 = _inv(w2 * masks[i])
                sub[i] = tj[ss] * np.sum(G * F1 * F2)
            total += sub if (m1, m2) == (0, 0) else 2 * np.real(sub)

    # ce:1063-1074: k3 bins
    k_center = 0.5 * (edges[1:] + edges[:-1])
    k3_edge = np.linspace(2 * k_min, 2 * k_max, 2 * k_bins + 1)[:-1]
    k3_center = 0.5 * (k3_edge[1:] + k3_edge[:-1])
    k3_bins = len(k3_center)
    k_num_k3, ksum3 = kbin_count(k3_bins, k3_edge, geo.knorm)
    k3_eff = ksum3 / k_num_k3
    full = data_vector_mode == "full"
    SN3_fft = None
    if tracer_type == "abc":
        SN0 = SN1 = SN2 = SN3 = 0.0
    else:
        SN0 = N_gal["a"] if (correlation_mode == "auto" and [l1, l2, L] == [0, 0, 0]) else 0.0
        other = ca if correlation_mode == "auto" else cb
        Pf = ca * np.conj(other) * V ** 2
        W_sn = None
        if correlation_mode == "auto":
            W_sn = compensation_kernel("bknoise", sampler, geo.w)
            Pf = Pf - SN0 * W_sn
        if L != 0:
            Pf = Pf * angular.ylm_function(L, 0, True)(*khat)
        tsum = radial_bin(Pf, k3_bins, k3_edge, geo.knorm)
        SN1, SN2 = 0.0, 0.0
        if l1 == L and l2 == 0:
            if correlation_mode == "auto":
                SN1 = (tsum / k_num_k3)[: len(k_center)] * (2 * L + 1)
                if l1 == 0:
                    SN2 = SN1.copy()
            elif tracer_type == "abb":
                SN1 = (tsum / k_num_k3)[: len(k_center)] * (2 * L + 1)
        if full:
            S1f = np.zeros((k_bins, k_bins), dtype="c16")
            S2f = np.zeros((k_bins, k_bins), dtype="c16")
            if np.ndim(SN1) == 0:
                S1f[:] = SN1
            else:
                for i in range(k_bins):
                    S1f[i, :] = SN1[i]
            if np.ndim(SN2) == 0:
                S2f[:] = SN2
            else:
                for i in range(k_bins):
                    S2f[:, i] = SN2[i]
            SN1, SN2 = S1f, S2f

        def s3_ana():
            # ce:1081-1180
            if tracer_type == "abb":
                return 0.0
            wk = k_num_k3 / k3_center
            if not full:
                s3 = np.zeros(k_bins, dtype="complex128")
                for i in range(k_bins):
                    q = angular.q_ells_eff(i, i, k_eff, l1, l2, L, k3_eff)
                    numer = np.sum(q * tsum / k3_center)
                    denom = np.sum(wk[: 2 * i + 1])
                    if denom > 0:
                        s3[i] = numer / denom
            else:
                s3 = np.zeros((k_bins, k_bins), dtype="complex128")
                for i in range(k_bins):
                    for j in range(k_bins):
                        q = angular.q_ells_eff(i, j, k_eff, l1, l2, L, k3_eff)
                        vb = angular.valid_k3_bins(k_center[i], k_center[j], k_min, k_max, k_bins)
                        numer = np.sum(q * tsum / k3_center)
                        denom = np.sum(wk * vb)
                        if denom > 0:
                            s3[i, j] = numer / denom
            return s3 * (H_ells * N_ells)

        def s3_fft():
            # ce:1182-1384
            if tracer_type == "abb":
                return np.zeros((k_bins, k_bins) if full else k_bins, dtype="complex128")
            src_c = ca * np.conj(other) * V ** 2
            if correlation_mode == "auto":
                src_c = src_c - SN0 * W_sn
            src = _inv(src_c)
            s3 = np.zeros((k_bins, k_bins) if full else k_bins, dtype="complex128")
            for ss, (m1, m2, _) in enumerate(cfgs):
                eq = l1 == l2 and m1 == m2
                cj = l1 == l2 and m1 == -m2
                yc1 = np.conj(angular.ylm_function(l1, m1, True)(*khat))
                yc2 = np.conj(angular.ylm_function(l2, m2, True)(*khat))
                use = sel if full else list(range(k_bins))
                S1 = {i: _inv(yc1 * masks[i]) for i in use}
                if eq:
                    S2 = S1
                elif cj:
                    S2 = {i: (-1) ** (m1 + l1) * np.conj(v) for i, v in S1.items()}
                else:
                    S2 = {i: _inv(yc2 * masks[i]) for i in use}
                if not full:
                    sub = np.zeros(k_bins, dtype="complex128")
                    for i in range(k_bins):
                        if k_num[i] > 0:
                            sub[i] = tj[ss] * np.sum(src * S1[i] * S2[i]) / k_num[i] ** 2
                else:
                    sub = np.zeros((k_bins, k_bins), dtype="complex128")
                    if bins is not None:
                        sub[:] = np.nan
                        for i in sel:
                            for j in sel:
                                sub[i, j] = 0.0
                    sym = eq or cj
                    for i in sel:
                        for j in sel:
                            if sym and j < i:
                                continue
                            if k_num[i] > 0 and k_num[j] > 0:
                                sub[i, j] = tj[ss] * np.sum(src * S1[i] * S2[j]) / (k_num[i] * k_num[j])
                    if sym:
                        for i in sel:
                            for j in sel:
                                if j > i:
                                    sub[j, i] = sub[i, j] if eq else np.conj(sub[i, j])
                s3 += sub if (m1, m2) == (0, 0) else 2.0 * np.real(sub)
            return s3 * (H_ells * N_ells) / N3

        if shotnoise_mode == "ana":
            SN3 = s3_ana()
        elif shotnoise_mode == "fft":
            SN3 = s3_fft()
        else:
            SN3 = s3_ana()
            SN3_fft = s3_fft()

    # ce:1495-1548
    Na = N_gal["a"]
    if correlation_mode == "auto":
        I_norm = Na ** 3 / V ** 2
    elif tracer_type == "aab":
        I_norm = Na ** 2 * N_gal["b"] / V ** 2
    elif tracer_type == "abb":
        I_norm = Na * N_gal["b"] ** 2 / V ** 2
    else:
        I_norm = Na * N_gal["b"] * N_gal["c"] / V ** 2
    shot = SN0 + SN1 + SN2 + SN3
    total = total * (N_ells * H_ells / I_norm)
    if full:
        total = total * (V ** 2 / np.outer(k_num, k_num))
    else:
        total = total * (V ** 2 / k_num ** 2)
    total = total * dV
    shot = shot * (1 / I_norm)
    sn_terms = {"SN0": SN0 / I_norm, "SN1": SN1 / I_norm, "SN2": SN2 / I_norm, "SN3": SN3 / I_norm}
    if shotnoise_mode == "both":
        sn_terms["SN3_FFT"] = SN3_fft / I_norm
    return {"B_sugi": total - shot, "SN_terms": sn_terms, "I_norm": I_norm,
            "Shot_noise": shot, "Bk_raw": total, "k_eff": k_eff, "nmodes": k_num}
