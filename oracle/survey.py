"""CPU restatement (numpy, complex128 full-spectrum fields) of CosmoNPC's survey path.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Survey fields are held
exactly as the reference holds them: complex128 "real" fields whose imaginary
part is the residue that the interlaced combination leaves on the Nyquist
planes (mesh_generator.py:207-219 followed by a complex-to-complex c2r).  That
residue reaches the survey multipoles through the x-space Y_lm weighting, so
it is kept.

Reference files: ``cp`` = src/cosmonpc/catalog_processor.py,
``mg`` = src/cosmonpc/mesh_generator.py, ``me`` = src/cosmonpc/math_evaluator.py,
``ce`` = src/cosmonpc/clustering_estimator.py.

The comoving distance uses the closed form of the flat LCDM integral,
  int_0^z dz'/E(z') = [F(1+z) - F(1)] / sqrt(1 - Om),
  F(x) = x 2F1(1/2, 1/3; 4/3; -Om x^3 / (1 - Om)),
a different method from the reference's (astropy) and from the device's
(Gauss-Legendre), which is the point of an independent check.
"""
from __future__ import annotations

import numpy as np
from scipy.special import hyp2f1

from . import angular
from .box import (KGeom, _fwd, _inv, compensation_kernel, kbin_count, paint_field,
                  radial_bin)
from .pmesh_lite import ParticleMesh

C_KMS = 299792.458


# ------------------------------------------------------------------ catalogs
def comoving_distance(z, h, omega_m):
    """Comoving distance in Mpc/h of flat LCDM without radiation (cp:617-632)."""
    z = np.asarray(z, dtype=np.float64)
    ol = 1.0 - omega_m
    a = omega_m / ol

    def F(x):
        return x * hyp2f1(0.5, 1.0 / 3.0, 4.0 / 3.0, -a * x ** 3)

    integral = (F(1.0 + z) - F(1.0)) / np.sqrt(ol)
    return integral * (C_KMS / (100.0 * h)) * h


def read_catalog(paths, column_names, z_range, comp_weight_plan, catalog_type, cosmology,
                 normalization_scheme):
    """``catalog_reader`` survey branch (cp:493-586): returns (cat dict, boxcenter)."""
    from cosmonpc_b200.fits import open_table

    assert "Z" in column_names
    parts = []
    for p in ([paths] if isinstance(paths, str) else paths):
        t = open_table(p)
        cols = [c for c in column_names if c in t.colnames()]
        parts.append(t.read_columns(cols))
    arr = np.concatenate(parts) if len(parts) > 1 else parts[0]
    if z_range is not None:
        arr = arr[(arr["Z"] > z_range[0]) & (arr["Z"] < z_range[1])]
    names = arr.dtype.names
    n = len(arr)
    # add_completeness_weight (cp:186-290)
    scheme, alias = comp_weight_plan["scheme"], comp_weight_plan["name_alias"]
    if "WEIGHT" in names:
        w = np.asarray(arr["WEIGHT"], dtype=np.float64)
    elif alias is None and scheme is None:
        w = np.ones(n)
    elif alias is not None and scheme is None:
        if alias not in names:
            raise ValueError(f"Alias {alias} not found in catalog columns.")
        w = np.asarray(arr[alias], dtype=np.float64)
    elif alias is None:
        if scheme == "boss":
            w = (arr["WEIGHT_SYSTOT"] * (arr["WEIGHT_NOZ"] + arr["WEIGHT_CP"] - 1.0)
                 if catalog_type == "data" else np.ones(n))
        elif scheme == "eboss":
            w = (arr["WEIGHT_SYSTOT"] * arr["WEIGHT_NOZ"] * arr["WEIGHT_CP"]
                 if catalog_type == "data" else np.ones(n))
        else:
            raise ValueError("DESI completeness weight scheme not yet implemented.")
    else:
        raise ValueError("Cannot specify both a scheme and an alias for completeness weight.")
    # ra_dec_z_to_xyz (cp:589-645)
    ra = np.deg2rad(arr["RA"])
    dec = np.deg2rad(arr["DEC"])
    if "Omega0" in cosmology:
        d = comoving_distance(arr["Z"], cosmology["h"], cosmology["Omega0"])
    else:  # cp:610-625: Planck18, then times the config's h
        from .cosmology import comoving_distance_mpc

        d = comoving_distance_mpc(arr["Z"]) * cosmology["h"]
    pos = np.column_stack([d * np.cos(dec) * np.cos(ra), d * np.cos(dec) * np.sin(ra), d * np.sin(dec)])
    if "WEIGHT_FKP" not in names:
        raise ValueError("WEIGHT_FKP column is missing in the catalog.")
    if "NZ" in names:
        nz = np.asarray(arr["NZ"], dtype=np.float64)
    elif "NX" in names:
        nz = np.asarray(arr["NX"], dtype=np.float64)
    elif normalization_scheme == "particle":
        raise ValueError("NZ column is missing in the catalog, which is required for particle normalization.")
    else:
        nz = np.ones(n)
    cat = {"pos": pos, "w": np.asarray(w, dtype=np.float64),
           "wfkp": np.asarray(arr["WEIGHT_FKP"], dtype=np.float64), "nz": nz}
    bc = 0.5 * (pos.min(axis=0) + pos.max(axis=0)) if n else np.zeros(3)
    return cat, bc


def subset(cat, mask):
    return {k: v[mask] for k, v in cat.items()}


# ------------------------------------------------------------ particle sums
def particle_sums_pk(data, randoms, correlation_mode):
    """``compute_particle_sums_pk`` (mg:1131-1190)."""
    wd, wr = data["w"] * data["wfkp"], randoms["w"] * randoms["wfkp"]
    out = [np.sum(wd), np.sum(wr), np.sum(data["w"]), np.sum(randoms["w"]),
           np.sum(data["w"] * data["nz"] * data["wfkp"] * data["wfkp"]),
           np.sum(randoms["w"] * randoms["nz"] * randoms["wfkp"] * randoms["wfkp"])]
    if correlation_mode == "auto":
        out += [np.sum(wd ** 2), np.sum(wr ** 2)]
    else:
        out += [0.0, 0.0]
    return out


def particle_sums_bk(data, randoms, correlation_mode, L):
    """``compute_particle_sums_bk`` (mg:1193-1268)."""
    wd, wr = data["w"] * data["wfkp"], randoms["w"] * randoms["wfkp"]
    I33 = np.sum(randoms["nz"] ** 2 * randoms["w"] ** 2 * randoms["wfkp"] ** 3)
    if correlation_mode == "auto":
        def s_lm(cat, wt):
            u = cat["pos"] / np.linalg.norm(cat["pos"], axis=1, keepdims=True)
            return np.array([np.sum(wt ** 3 * np.conj(angular.ylm_function(L, M, True)(u[:, 0], u[:, 1], u[:, 2])))
                             for M in range(L + 1)])
        sd, sr = s_lm(data, wd), s_lm(randoms, wr)
    else:
        sd = sr = 0.0
    return [np.sum(wd), np.sum(wr), np.sum(data["w"]), np.sum(randoms["w"]), I33, sd, sr]


# ------------------------------------------------------------------ meshes
class Cfg:
    """The config keys the survey path reads, with the reference's defaults."""

    def __init__(self, c):
        self.c = c
        self.n = int(c["nmesh"][0])
        self.L = float(c["boxsize"][0])
        self.sampler = c["sampler"]
        self.interlaced = bool(c["interlaced"])
        self.dV = self.L ** 3 / self.n ** 3

    def read(self, key, catalog_type, bc=None):
        c = self.c
        return read_catalog(c["catalogs"][key], c["column_names"], c["z_range"], c["comp_weight_plan"],
                            catalog_type, c["cosmology"], c.get("normalization_scheme", "particle"))

    def paint(self, cat, weight, bc):
        return paint_field(cat["pos"] - bc, weight, self.n, self.L, self.sampler, self.interlaced)


def alpha_of(sums, scheme):
    if scheme == "pypower":
        return sums[0] / sums[1]
    if scheme == "nbodykit":
        return sums[2] / sums[3]
    raise ValueError("alpha_scheme must be either 'pypower' or 'nbodykit'.")


def mesh_pk_survey(c):
    """``get_mesh_pk_survey`` (mg:227-538): (attrs, field_a, field_b)."""
    cfg = Cfg(c)
    corr = c["correlation_mode"]
    norm = c["normalization_scheme"]
    ascheme = c.get("alpha_scheme", "pypower")
    ra_, bc = cfg.read("randoms_a", "randoms")
    da_, _ = cfg.read("data_a", "data")
    s = particle_sums_pk(da_, ra_, corr)
    alpha_a = alpha_of(s, ascheme)
    attrs = {"boxcenter": bc, "alpha_a": alpha_a, "I_rand": alpha_a * s[5], "I_data": s[4]}
    Da = cfg.paint(da_, da_["w"] * da_["wfkp"], bc) / cfg.dV
    Ra = cfg.paint(ra_, ra_["w"] * ra_["wfkp"], bc) / cfg.dV
    fa = Da - alpha_a * Ra
    fb = fa
    if corr == "cross":
        db_, _ = cfg.read("data_b", "data")
        rb_, _ = cfg.read("randoms_b", "randoms")
        sb = particle_sums_pk(db_, rb_, corr)
        alpha_b = alpha_of(sb, ascheme)
        attrs["alpha_b"] = alpha_b
        Db = cfg.paint(db_, db_["w"] * db_["wfkp"], bc) / cfg.dV
        Rb = cfg.paint(rb_, rb_["w"] * rb_["wfkp"], bc) / cfg.dV
        fb = Db - alpha_b * Rb
    if norm == "particle":
        if corr != "auto":
            raise ValueError("Particle-normalization scheme will not work for cross-correlation!")
        attrs["N0"] = (s[6] + alpha_a ** 2 * s[7]) / attrs["I_rand"]
    else:
        if corr == "auto":
            I = alpha_a * np.sum(Da * Ra) * cfg.L ** 3 / cfg.n ** 3
        else:
            I = 0.5 * cfg.L ** 3 / cfg.n ** 3 * (attrs["alpha_b"] * np.sum(Da * Rb) + alpha_a * np.sum(Db * Ra))
        I = np.float64(np.real(I))
        attrs["I_mesh"] = I
        attrs["N0"] = (s[6] + alpha_a ** 2 * s[7]) / I if corr == "auto" else 0.0
    return attrs, fa, fb


def xgrid(n, L, bc):
    """``get_xgrid`` (me:25-32): unit vectors of the cell positions."""
    pm = ParticleMesh([L] * 3, [n] * 3)
    off = 0.5 * np.array([L] * 3) / np.array([n] * 3) + np.asarray(bc)
    xs = [np.broadcast_to(pm.x[i] + off[i], (n, n, n)) for i in range(3)]
    xn = np.sqrt(sum(x ** 2 for x in xs))
    return [x / xn for x in xs]


def _flip(a):
    """k -> -k index map (me:619-630): index 0 fixed, the rest reversed, per axis."""
    out = a
    for ax in range(3):
        out = np.roll(np.flip(out, axis=ax), 1, axis=ax)
    return out


# ------------------------------------------------------------- pk survey
def pk_survey(c, attrs, fa, fb):
    """``calculate_power_spectrum_survey`` (ce:205-563) with ``get_G_ell`` (ce:3104-3134)."""
    cfg = Cfg(c)
    corr = c["correlation_mode"]
    poles = c["poles"]
    mode = c.get("high_order_mode", "default")
    n, L = cfg.n, cfg.L
    V = L ** 3
    I = attrs["I_rand"] if c["normalization_scheme"] == "particle" else attrs["I_mesh"]
    N0 = attrs["N0"]
    edges = np.linspace(c["k_min"], c["k_max"], c["k_bins"] + 1)
    kb = c["k_bins"]
    geo = KGeom(n, L)
    kind = "sinc" if cfg.interlaced else "shotnoise"
    comp = compensation_kernel(kind, cfg.sampler, geo.w)
    ca = _fwd(fa) * comp * V
    cb = ca if corr == "auto" else _fwd(fb) * comp * V
    xg = xgrid(n, L, attrs["boxcenter"]) if poles != [0] else None
    k_num, ksum = kbin_count(kb, edges, geo.knorm)
    res = {"k_eff": ksum / k_num, "k_num": k_num, "I_norm": I}

    strat = None
    if mode != "default" and corr == "auto" and poles in ([0, 2, 4], [0, 2, 4, 6], [0, 2, 4, 6, 8]):
        high = {p for p in poles if p in (4, 6, 8)}
        if mode == "fast":
            fast = {(0, 2, 4): {4}, (0, 2, 4, 6): {6}, (0, 2, 4, 6, 8): {6, 8}}[tuple(poles)]
            exact = {(0, 2, 4): set(), (0, 2, 4, 6): {4}, (0, 2, 4, 6, 8): {4}}[tuple(poles)]
        else:
            fast, exact = high, high
        internal = {4} if (fast & {6, 8}) else set()
        strat = {"fast": fast, "exact": exact | internal, "visible": exact,
                 "f2": bool(fast & {4, 6, 8}), "f4": bool(fast & {6, 8})}
    F2 = F4 = None

    def G_ell(ell):
        Y = [angular.ylm_function(ell, m) for m in range(ell + 1)]
        G = _fwd(fb_field * Y[0](*xg)) * Y[0](*geo.khat)
        for m in range(1, ell + 1):
            G = G + 2 * (_fwd(fb_field * np.conj(Y[m](*xg))) * Y[m](*geo.khat))
        return G * comp * (4 * np.pi * V / (2 * ell + 1))

    fb_field = fb
    for pole in poles:
        if pole == 0:
            P = np.real(ca) ** 2 + np.imag(ca) ** 2 if corr == "auto" else ca * np.conj(cb)
        else:
            store = True
            if pole in (4, 6, 8) and strat is not None:
                store = pole in strat["exact"]
            c2 = pole == 2 and strat is not None and strat["f2"]
            c4 = pole == 4 and strat is not None and strat["f4"]
            if not (store or c2 or c4):
                continue
            G = G_ell(pole)
            if c2:
                F2 = 0.5 * (G + np.conj(_flip(G)))
            if c4:
                F4 = 0.5 * (G + np.conj(_flip(G)))
            if not store:
                continue
            P = ca * np.conj(G)
        r = radial_bin(P, kb, edges, geo.knorm) / k_num
        r = r * ((2 * pole + 1) / I)
        if pole == 0:
            r = r - N0
        else:
            r = np.imag(r) if pole & 1 else np.real(r)
        res[f"P{pole}"] = r
    if strat is not None and strat["fast"]:
        if 4 in strat["fast"]:
            P22 = radial_bin(F2 * np.conj(F2), kb, edges, geo.knorm) / k_num * (9 / I) - N0 * 9 / 5
            res["P4b"] = np.real(35 / 18 * P22 - res["P2"] - 7 / 2 * res["P0"])
        if strat["fast"] & {6, 8}:
            s42 = radial_bin(F4 * np.conj(F2), kb, edges, geo.knorm)
            if 6 in strat["fast"]:
                P42 = s42 / k_num * (13 / I)
                res["P6b"] = np.real(11 / 5 * P42 - 52 / 63 * res["P4"] - 286 / 175 * res["P2"])
            if 8 in strat["fast"]:
                P42 = s42 / k_num * (13 / I)
                P44 = radial_bin(F4 * np.conj(F4), kb, edges, geo.knorm) / k_num * (17 / I) - N0 * 17 / 9
                res["P8b"] = np.real(1287 / 490 * P44 - 374 / 245 * P42 - 3553 / 15435 * res["P4"]
                                     - 1326 / 8575 * res["P2"] - 2431 / 490 * res["P0"])
        if mode == "fast":
            for p in strat["fast"]:
                res.pop(f"P{p}", None)
    return res


# ------------------------------------------------------------- bk meshes
def mesh_bk_survey(c):
    """``get_mesh_bk_survey`` (mg:541-1004): (attrs, fields {a, b, c}, caches)."""
    cfg = Cfg(c)
    corr = c["correlation_mode"]
    tt = c["tracer_type"]
    L_ = c["angu_config"][2]
    norm = c.get("normalization_scheme", "particle")
    ascheme = c.get("alpha_scheme", "pypower")
    _, bc = cfg.read("randoms_a", "randoms")
    attrs = {"normalization_scheme": norm, "boxcenter": bc}
    cache = {}

    def prep(label):
        r_, _ = cfg.read(f"randoms_{label}", "randoms")
        d_, _ = cfg.read(f"data_{label}", "data")
        s = particle_sums_bk(d_, r_, corr, L_)
        alpha = alpha_of(s, ascheme)
        attrs[f"alpha_{label}"] = alpha
        attrs[f"I_33_{label}"] = s[4] * alpha
        attrs[f"S_LM_{label}"] = s[5] - alpha ** 3 * s[6]
        D = cfg.paint(d_, d_["w"] * d_["wfkp"], bc) * (1 / cfg.dV)
        R = cfg.paint(r_, r_["w"] * r_["wfkp"], bc) * (alpha / cfg.dV)
        cache[label] = (D, R)
        return D - R

    fields = {"a": prep("a"), "b": None, "c": None}
    if corr == "cross":
        fields["b"] = prep("b")
        if tt == "abc":
            fields["c"] = prep("c")
    dV = cfg.dV
    if norm == "particle":
        assert corr == "auto"
        attrs["I_norm"] = attrs["I_33_a"]
    elif norm == "mesh":
        assert corr == "auto"
        attrs["I_norm"] = dV * np.sum(cache["a"][1] ** 3)
    else:
        if corr == "auto":
            D = cache["a"][0]
            d_, _ = cfg.read("data_a", "data")
            r_, _ = cfg.read("randoms_a", "randoms")
            odd = np.arange(r_["pos"].shape[0]) % 2 == 1
            ro, re_ = subset(r_, odd), subset(r_, ~odd)
            if ascheme == "pypower":
                sd = np.sum(d_["w"] * d_["wfkp"])
                so, se = np.sum(ro["w"] * ro["wfkp"]), np.sum(re_["w"] * re_["wfkp"])
            elif ascheme == "nbodykit":
                sd, so, se = np.sum(d_["w"]), np.sum(ro["w"]), np.sum(re_["w"])
            else:
                raise ValueError("alpha_scheme must be either 'pypower' or 'nbodykit'.")
            Ro = cfg.paint(ro, ro["w"] * ro["wfkp"], bc) * ((sd / so) / dV)
            Re = cfg.paint(re_, re_["w"] * re_["wfkp"], bc) * ((sd / se) / dV)
            attrs["I_norm"] = dV * np.sum(D * Ro * Re)
        else:
            if tt == "abc":
                I = dV * np.sum(cache["a"][1] * cache["b"][1] * cache["c"][1])
            elif tt == "aab":
                I = dV * np.sum(cache["a"][0] * cache["a"][1] * cache["b"][1])
            else:  # abb
                I = dV * np.sum(cache["a"][1] * cache["b"][1] * cache["b"][0])
            attrs["I_norm"] = I
    return attrs, fields


def n_field(c, label, alpha, bc):
    """``get_N_field`` (mg:1007-1128)."""
    cfg = Cfg(c)
    r_, _ = cfg.read(f"randoms_{label}", "randoms")
    d_, _ = cfg.read(f"data_{label}", "data")
    D = cfg.paint(d_, (d_["w"] * d_["wfkp"]) ** 2, bc) / cfg.dV
    R = cfg.paint(r_, (r_["w"] * r_["wfkp"]) ** 2, bc) / cfg.dV
    return D + alpha ** 2 * R


# ------------------------------------------------------------- bk survey
def bk_survey(c, attrs, fields):
    """``calculate_bk_sugi_survey`` (ce:1558-3101): the result dict (results only)."""
    cfg = Cfg(c)
    corr = c["correlation_mode"]
    tt = c["tracer_type"]
    dvm = c.get("data_vector_mode", "diagonal")
    snm = c.get("shotnoise_mode", "ana")
    bs = c.get("block_size", 1 if dvm == "diagonal" else "full")
    l1, l2, L = c["angu_config"]
    n, Lb = cfg.n, cfg.L
    V = Lb ** 3
    N3 = float(n) ** 3
    dV = cfg.dV
    I = attrs["I_norm"]
    kmin, kmax, kb = c["k_min"], c["k_max"], c["k_bins"]
    N_ells = (2 * l1 + 1) * (2 * l2 + 1) * (2 * L + 1)
    H_ells = angular.wigner3j(l1, l2, L, 0, 0, 0)
    cfgs, tj = angular.magnetic_configs_survey(l1, l2, L)
    edges = np.linspace(kmin, kmax, kb + 1)
    geo = KGeom(n, Lb)
    comp = compensation_kernel("sinc", cfg.sampler, geo.w)
    csn = compensation_kernel("bknoise", cfg.sampler, geo.w)
    fa, fb, fc = fields["a"], fields["b"], fields["c"]
    ca = _fwd(fa) * comp * V
    cb = ca if corr == "auto" else _fwd(fb) * comp * V
    kh = geo.khat
    xg = xgrid(n, Lb, attrs["boxcenter"])
    k_num, ksum = kbin_count(kb, edges, geo.knorm)
    k_eff = ksum / k_num
    f3 = fa if corr == "auto" else (fc if tt == "abc" else fb)
    masks = [np.logical_and(geo.knorm >= edges[i], geo.knorm < edges[i + 1]) for i in range(kb)]
    idx = {cf: i for i, cf in enumerate(cfgs)}
    same12 = corr == "auto" or tt == "aab"
    same_l = l1 == l2

    def G_of(M):
        return _inv(_fwd(f3 * angular.ylm_function(L, M, True)(*xg)) * comp)

    done = set()
    curM, G = None, None
    full = dvm == "full"
    total = np.zeros((kb, kb) if full else kb, dtype=np.complex128)
    if full:
        bs = kb if bs == "full" else bs
        if not (isinstance(bs, int) and 1 <= bs <= kb):
            raise ValueError("For full mode, block_size must be 1, 'full', or an integer in [1, k_bins].")
    for ss, (m1, m2, M) in enumerate(cfgs):
        if (m1, m2, M) in done:
            continue
        if M != curM:
            G, curM = G_of(M), M
        w1 = ca * angular.ylm_function(l1, m1, True)(*kh)
        eq = same12 and same_l and m1 == m2
        cj = same12 and same_l and m1 == -m2
        src2 = ca if tt in ("aaa", "aab") else cb
        w2 = src2 * angular.ylm_function(l2, m2, True)(*kh)
        F1 = [_inv(w1 * mk) for mk in masks]
        if full:
            sub = np.zeros((kb, kb), dtype=np.complex128)
            for i in range(kb):
                for j in range(kb):
                    if (eq or cj) and j < i:
                        continue
                    if eq:
                        F2 = F1[j]
                    elif cj:
                        F2 = (-1) ** (m1 + l1) * np.conj(F1[j])
                    else:
                        F2 = _inv(w2 * masks[j])
                    sub[i, j] = tj[ss] * np.sum(G * F1[i] * F2)
            if eq or cj:
                for i in range(kb):
                    for j in range(i + 1, kb):
                        sub[j, i] = sub[i, j] if eq else np.conj(sub[i, j])
        else:
            sub = np.zeros(kb, dtype=np.complex128)
            for i in range(kb):
                if eq:
                    F2 = F1[i]
                elif cj:
                    F2 = (-1) ** (m1 + l1) * np.conj(F1[i])
                else:
                    F2 = _inv(w2 * masks[i])
                sub[i] = tj[ss] * np.sum(G * F1[i] * F2)
        swap = (m2, m1, M)
        add_swap = same12 and same_l and swap in idx and swap != (m1, m2, M) and swap not in done
        if add_swap:
            sub = sub + sub.T if full else 2.0 * sub
        total += sub if (m1, m2, M) == (0, 0, 0) else 2 * np.real(sub)
        if add_swap:
            done.add(swap)
        done.add((m1, m2, M))

    # shot noise (ce:2070-3077)
    k_center = 0.5 * (edges[1:] + edges[:-1])
    k3_edge = np.linspace(2 * kmin, 2 * kmax, kb * 2 + 1)[:-1]
    k3_center = 0.5 * (k3_edge[1:] + k3_edge[:-1])
    k3b = len(k3_center)
    k_num3, ks3 = kbin_count(k3b, k3_edge, geo.knorm)
    k3_eff = ks3 / k_num3
    shape = (kb, kb) if full else (kb,)
    SN0 = 0.0 + 0.0j
    SN1 = np.zeros(shape, dtype="c16")
    SN2 = np.zeros(shape, dtype="c16")
    SN3 = np.zeros(shape, dtype="c16")
    SN3f = None
    if tt != "abc":
        if tt == "aab":
            rshot, Nshot, S_LM = fb, n_field(c, "a", attrs["alpha_a"], attrs["boxcenter"]), attrs.get("S_LM_a")
        elif tt == "abb":
            rshot, Nshot, S_LM = fa, n_field(c, "b", attrs["alpha_b"], attrs["boxcenter"]), attrs.get("S_LM_b")
        else:
            rshot, Nshot, S_LM = fa, n_field(c, "a", attrs["alpha_a"], attrs["boxcenter"]), attrs.get("S_LM_a")
        sbar = corr == "auto" and tt == "aaa"
        S_arr = None
        if sbar:
            S_arr = (np.zeros(L + 1, "c16") if S_LM is None else
                     (np.concatenate([[S_LM], np.zeros(L, "c16")]) if np.isscalar(S_LM)
                      else np.asarray(S_LM, dtype="c16")))
        if tt == "aaa" and [l1, l2, L] == [0, 0, 0]:
            S = attrs.get("S_LM_a", 0.0)
            SN0 = S[0] if isinstance(S, np.ndarray) else S
        if tt in ("aaa", "abb") and l1 == L and l2 == 0:
            cd = _fwd(rshot) * comp * V
            acc = np.zeros_like(cd)
            for M in range(L + 1):
                y = angular.ylm_function(L, M, True)
                cN = _fwd(Nshot * y(*xg)) * comp * V
                term = cd * np.conj(cN)
                if sbar:
                    term = term - S_arr[M] * csn
                acc += (0.5 if M == 0 else 1.0) * (term * y(*kh))
            tot = 2.0 * np.real(radial_bin(acc, kb, edges, geo.knorm))
            v = np.zeros(kb, dtype="c16")
            ok = k_num > 0
            v[ok] = (2 * L + 1) * tot[ok] / k_num[ok]
            if full:
                for i in range(kb):
                    SN1[i, :] = v[i]
            else:
                SN1 = v
            if tt == "aaa" and [l1, l2, L] == [0, 0, 0]:
                if full:
                    for i in range(kb):
                        SN2[:, i] = v[i]
                else:
                    SN2 = v.copy()
        if tt != "abb":
            cN00 = _fwd(Nshot) * comp * V

            def delta_lm(M):
                return _fwd(rshot * np.conj(angular.ylm_function(L, M, True)(*xg))) * comp * V

            def ana():
                acc = np.zeros_like(cN00)
                for M in range(L + 1):
                    term = delta_lm(M) * np.conj(cN00)
                    if sbar:
                        term = term - S_arr[M] * csn
                    acc += (0.5 if M == 0 else 1.0) * (term * angular.ylm_function(L, M, True)(*kh))
                Q = (2.0 * np.real(radial_bin(acc, k3b, k3_edge, geo.knorm))).astype("c16")
                wk = np.zeros(k3b)
                ok = k_num3 > 0
                wk[ok] = k_num3[ok] / k3_center[ok]
                out = np.zeros(shape, dtype="c16")
                if not full:
                    for i in range(kb):
                        q = angular.q_ells_eff(i, i, k_eff, l1, l2, L, k3_eff)
                        den = np.sum(wk[: 2 * i + 1])
                        if den > 0:
                            out[i] = np.sum(q * Q / k3_center) / den
                else:
                    for i in range(kb):
                        for j in range(kb):
                            q = angular.q_ells_eff(i, j, k_eff, l1, l2, L, k3_eff)
                            vb = angular.valid_k3_bins(k_center[i], k_center[j], kmin, kmax, kb)
                            den = np.sum(wk * vb)
                            if den > 0:
                                out[i, j] = np.sum(q * Q / k3_center) / den
                return out * (H_ells * N_ells)

            def fft():
                def s_val(Mi):
                    if S_arr is None:
                        return 0.0 + 0.0j
                    return S_arr[Mi] if Mi >= 0 else ((-1) ** Mi) * np.conj(S_arr[-Mi])

                def shell(ell, m, b):
                    return _inv(np.conj(angular.ylm_function(ell, m, True)(*kh)) * masks[b])

                out = np.zeros(shape, dtype="c16")
                dn = set()
                curM2, src = None, None
                for ss, (m1, m2, M) in enumerate(cfgs):
                    if (m1, m2, M) in dn:
                        continue
                    if M != curM2:
                        sf = delta_lm(M) * np.conj(cN00)
                        if sbar:
                            sf = sf - s_val(M) * csn
                        src, curM2 = _inv(sf), M
                    eq = l1 == l2 and m1 == m2
                    cj = l1 == l2 and m1 == -m2
                    if not full:
                        sub = np.zeros(kb, dtype="c16")
                        for i in range(kb):
                            s1 = shell(l1, m1, i)
                            s2 = s1 if eq else ((-1) ** (m1 + l1) * np.conj(s1) if cj else shell(l2, m2, i))
                            if k_num[i] > 0:
                                sub[i] = tj[ss] * np.sum(s1 * s2 * src) / k_num[i] ** 2
                    else:
                        sub = np.zeros((kb, kb), dtype="c16")
                        for i in range(kb):
                            s1 = shell(l1, m1, i)
                            for j in range(kb):
                                if (eq or cj) and j < i:
                                    continue
                                if eq:
                                    s2 = shell(l1, m1, j)
                                elif cj:
                                    s2 = (-1) ** (m1 + l1) * np.conj(shell(l1, m1, j))
                                else:
                                    s2 = shell(l2, m2, j)
                                if k_num[i] > 0 and k_num[j] > 0:
                                    sub[i, j] = tj[ss] * np.sum(s1 * s2 * src) / (k_num[i] * k_num[j])
                        if eq or cj:
                            for i in range(kb):
                                for j in range(i + 1, kb):
                                    sub[j, i] = sub[i, j] if eq else np.conj(sub[i, j])
                    swap = (m2, m1, M)
                    add_swap = l1 == l2 and swap in idx and swap != (m1, m2, M) and swap not in dn
                    if add_swap:
                        sub = 2.0 * sub if not full else sub + sub.T
                    out += sub if (m1, m2, M) == (0, 0, 0) else 2.0 * np.real(sub)
                    if add_swap:
                        dn.add(swap)
                    dn.add((m1, m2, M))
                return out * (H_ells * N_ells) / N3

            if snm == "both":
                SN3, SN3f = ana(), fft()
            elif snm == "ana":
                SN3 = ana()
            else:
                SN3 = fft()
        elif snm == "both":
            SN3f = np.zeros(shape, dtype="c16")
    elif snm == "both":
        SN3f = None
    total = total * (N_ells * H_ells / I)
    total = total * (1.0 / np.outer(k_num, k_num) if full else 1.0 / k_num ** 2)
    total = total * dV
    shot = (SN0 + SN1 + SN2 + SN3) / I
    sn = {"SN0": SN0 / I, "SN1": SN1 / I, "SN2": SN2 / I, "SN3": SN3 / I}
    if snm == "both":
        sn["SN3_FFT"] = SN3f / I
    return {"B_sugi": total - shot, "Bk_raw": total, "SN_terms": sn, "Shot_noise": shot,
            "I_norm": I, "k_eff": k_eff, "nmodes": k_num}


def run_survey(config):
    """Survey branch of ``run_task`` (te:44-147, te:219-317) without the file output."""
    c = dict(config)
    if c["statistic"] == "pk":
        attrs, fa, fb = mesh_pk_survey(c)
        res = pk_survey(c, attrs, fa, fb)
    else:
        c.setdefault("block_size", 1 if c.get("data_vector_mode", "diagonal") == "diagonal" else "full")
        attrs, fields = mesh_bk_survey(c)
        res = bk_survey(c, attrs, fields)
    res.update(attrs)
    return res
