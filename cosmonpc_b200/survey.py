"""Survey-geometry path on the device: catalogs, FKP fields, normalisations and
the survey power-spectrum / Sugiyama-bispectrum estimators.

Drop-in for the reference's ``get_mesh_pk_survey`` / ``get_mesh_bk_survey`` /
``get_N_field`` / ``compute_particle_sums_*`` (src/cosmonpc/mesh_generator.py:227-1268),
the survey branch of ``catalog_reader`` (src/cosmonpc/catalog_processor.py:446-645),
``calculate_power_spectrum_survey`` with ``get_G_ell``
(src/cosmonpc/clustering_estimator.py:205-563, :3104-3134) and
``calculate_bk_sugi_survey`` (clustering_estimator.py:1558-3101).  Same config
keys, result dictionaries and errors.

Field representation.  The reference holds each painted field as a complex128
"real" field; with interlacing its imaginary part is the residue of the
non-Hermitian Nyquist planes of s1/2 + s2/2 e^{i k.H/2}.  That residue reaches
the survey multipoles through the x-space Y_lm weighting (at the 1e-3 level),
so a :class:`SurveyField` carries it as a second real field.

Every per-particle, per-cell and per-mode operation runs in libcosmonpc_b200.so
(or cuFFT); the host does O(k_bins^2) algebra only.
"""
from __future__ import annotations

import logging
import os

import numpy as np
import torch

from . import _lib, angular, engine
from .catalog_processor import SUPPORTED, _ext
from .fits import open_table

log = logging.getLogger("cosmonpc_b200")


def _device():
    return engine._device()


# ================================================================ catalogs
class SurveyCatalog:
    """A decoded survey catalog on the device (positions in Mpc/h, FP64)."""

    def __init__(self, pos, w, wfkp, nz):
        self.pos, self.w, self.wfkp, self.nz = pos, w, wfkp, nz
        self.n = int(pos.shape[0])

    def take(self, sl):
        return SurveyCatalog(self.pos[sl].contiguous(), self.w[sl].contiguous(), self.wfkp[sl].contiguous(),
                             self.nz[sl].contiguous())

    def paint_weights(self, power=1):
        """(WEIGHT * WEIGHT_FKP)^power on the device."""
        out = torch.empty(self.n, dtype=torch.float64, device=self.pos.device)
        if self.n:
            _lib.Context.get().catalog_weights(self.n, self.w, self.wfkp, power, out)
        return out


# decoded catalogs of one run_stats call, keyed by every input that shapes them
# (the reference re-reads a file each time a stage needs it; the result is the same)
_cache = {}


def clear_cache():
    _cache.clear()


def _weight_rule(names, comp_weight_plan, catalog_type):
    """add_completeness_weight (catalog_processor.py:186-290) decided on the host."""
    scheme = comp_weight_plan["scheme"]
    alias = comp_weight_plan["name_alias"]
    assert catalog_type in ["data", "randoms"], "catalog_type must be 'data' or 'randoms'"
    assert scheme in [None, "boss", "eboss", "desi"]
    if "WEIGHT" in names:
        return _lib.W_COLUMN, "WEIGHT"
    if alias is None and scheme is None:
        return _lib.W_ONE, None
    if alias is not None and scheme is None:
        if alias in names:
            return _lib.W_COLUMN, alias
        raise ValueError(f"Alias {alias} not found in catalog columns.")
    if alias is None and scheme is not None:
        if scheme == "boss":
            return (_lib.W_BOSS if catalog_type == "data" else _lib.W_ONE), None
        if scheme == "eboss":
            return (_lib.W_EBOSS if catalog_type == "data" else _lib.W_ONE), None
        raise ValueError("DESI completeness weight scheme not yet implemented.")
    raise ValueError("Cannot specify both a scheme and an alias for completeness weight.")


def _column(table, name):
    c = table.scalar_column(name)
    col = _lib.Column()
    col.type = _lib.CT_OF_FITS[c.code]
    col.offset = c.offset
    col.scale = c.scale
    col.zero = c.zero
    return col


_COPY_THREADS = max(1, min(8, os.cpu_count() or 1))


def _parallel_copy(dst, src):
    """dst[:] = src for (rows, bytes) arrays, row blocks copied by a thread pool."""
    n = src.shape[0]
    if n < 65536 or _COPY_THREADS == 1:
        np.copyto(dst, src)
        return
    from concurrent.futures import ThreadPoolExecutor

    cuts = np.linspace(0, n, _COPY_THREADS + 1).astype(np.int64)
    with ThreadPoolExecutor(_COPY_THREADS) as ex:
        list(ex.map(lambda i: np.copyto(dst[cuts[i]:cuts[i + 1]], src[cuts[i]:cuts[i + 1]]),
                    range(_COPY_THREADS)))


def _decode_file(path, column_names, z_range, comp_weight_plan, catalog_type, cosmology,
                 normalization_scheme):
    t = open_table(path)
    names = [c for c in column_names if c in t.colnames()]
    for req in ("RA", "DEC", "Z"):
        if req not in names:
            raise ValueError(f"no field of name {req}")
    rule, wcol = _weight_rule(names, comp_weight_plan, catalog_type)
    spec = _lib.CatalogSpec()
    spec.row_bytes = t.row_bytes
    for slot in range(_lib.NCOLS):
        spec.col[slot].type = _lib.CT_ABSENT
    spec.col[_lib.COL_RA] = _column(t, "RA")
    spec.col[_lib.COL_DEC] = _column(t, "DEC")
    spec.col[_lib.COL_Z] = _column(t, "Z")
    if rule == _lib.W_COLUMN:
        spec.col[_lib.COL_WEIGHT] = _column(t, wcol)
    elif rule in (_lib.W_BOSS, _lib.W_EBOSS):
        for slot, nm in ((_lib.COL_SYSTOT, "WEIGHT_SYSTOT"), (_lib.COL_NOZ, "WEIGHT_NOZ"),
                         (_lib.COL_CP, "WEIGHT_CP")):
            if nm not in names:
                raise ValueError(f"no field of name {nm}")
            spec.col[slot] = _column(t, nm)
    spec.weight_rule = rule
    if "WEIGHT_FKP" not in names:
        raise ValueError("WEIGHT_FKP column is missing in the catalog.")
    spec.col[_lib.COL_FKP] = _column(t, "WEIGHT_FKP")
    if "NZ" in names:
        spec.col[_lib.COL_NZ] = _column(t, "NZ")
    elif "NX" in names:
        spec.col[_lib.COL_NZ] = _column(t, "NX")
    elif normalization_scheme == "particle":
        raise ValueError("NZ column is missing in the catalog, which is required for particle normalization.")
    spec.has_zrange = 0 if z_range is None else 1
    if z_range is not None:
        spec.z_min, spec.z_max = float(z_range[0]), float(z_range[1])
    spec.h = float(cosmology["h"])
    if "Omega0" in cosmology:
        spec.omega_m = float(cosmology["Omega0"])
        spec.cosmology = _lib.COSMO_FLAT_LCDM
    else:  # catalog_processor.py:610-625: Planck18, distances still times the config's h
        spec.omega_m = 0.0
        spec.cosmology = _lib.COSMO_PLANCK18
    dev = _device()
    nr = t.nrows
    # file rows -> one pinned buffer (a single host copy, split over threads:
    # numpy releases the GIL for the copy) -> device
    raw = t.rows()
    host = torch.empty(raw.size, dtype=torch.uint8, pin_memory=True)
    if raw.size:
        _parallel_copy(host.numpy().reshape(raw.shape), raw)
    rows = host.to(dev, non_blocking=True)
    del raw, host
    cap = max(nr, 1)
    pos = torch.empty((cap, 3), dtype=torch.float64, device=dev)
    w = torch.empty(cap, dtype=torch.float64, device=dev)
    wf = torch.empty(cap, dtype=torch.float64, device=dev)
    nz = torch.empty(cap, dtype=torch.float64, device=dev)
    kept = _lib.Context.get().catalog_decode(rows, nr, spec, pos, w, wf, nz)
    del rows
    return pos[:kept], w[:kept], wf[:kept], nz[:kept]


def read_catalog(catalog, column_names, z_range, comp_weight_plan, catalog_type, cosmology,
                 normalization_scheme="particle"):
    """Survey branch of ``catalog_reader`` (catalog_processor.py:446-586) on the device."""
    ext = _ext(catalog)
    if ext not in SUPPORTED:
        raise ValueError(f"Unsupported data file type: {ext}")
    if ext == "npy":
        raise NotImplementedError("Survey-like geometry with .npy file is not yet implemented.")
    if ext != "fits":
        raise NotImplementedError("survey-like catalogs are read from .fits files")
    assert "Z" in column_names, \
        "For survey-like geometry with .fits file, column_names must include 'Z' for redshift slice."
    # the reference falls back to Planck18 when h or Omega0 is missing
    # (catalog_processor.py:610-625) and then multiplies by cosmology["h"]:
    # without a config dict, or without h, it fails there
    if cosmology is None:
        raise TypeError("'NoneType' object is not subscriptable")
    if "h" not in cosmology:
        raise KeyError("h")
    paths = [catalog] if isinstance(catalog, str) else list(catalog)
    key = (tuple(paths), tuple(column_names), None if z_range is None else tuple(z_range),
           comp_weight_plan["scheme"], comp_weight_plan["name_alias"], catalog_type,
           float(cosmology["h"]), float(cosmology.get("Omega0", -1.0)), normalization_scheme == "particle",
           torch.cuda.current_device())
    hit = _cache.get(key)
    if hit is not None:
        return hit
    parts = [_decode_file(p, column_names, z_range, comp_weight_plan, catalog_type, cosmology,
                          normalization_scheme) for p in paths]
    if len(parts) == 1:
        cat = SurveyCatalog(*parts[0])
    else:
        cat = SurveyCatalog(*[torch.cat([p[i] for p in parts]) for i in range(4)])
    _cache[key] = cat
    return cat


class ParticleSums:
    """compute_particle_sums_pk / _bk (mesh_generator.py:1131-1268) of one catalog."""

    def __init__(self, cat, L=None):
        nh = 0 if L is None else L + 1
        harms = [angular.harmonic(L, M, True) for M in range(nh)]
        out = torch.empty(_lib.PSUM_COUNT + 2 * nh + 6, dtype=torch.float64, device=cat.pos.device)
        _lib.Context.get().particle_sums(cat.n, cat.pos, cat.w, cat.wfkp, cat.nz, harms, out)
        v = out.cpu().numpy()
        self.w_wfkp, self.w, self.I_sum, self.N_sum, self.I33 = (float(x) for x in v[:5])
        self.S_LM = v[5:5 + 2 * nh:2] + 1j * v[6:6 + 2 * nh:2] if nh else 0.0
        self.lo = v[5 + 2 * nh:8 + 2 * nh]
        self.hi = v[8 + 2 * nh:11 + 2 * nh]


def boxcenter_of(sums):
    """catalog_reader's boxcenter = 0.5 (min + max) of the positions (cp:564-574)."""
    return 0.5 * (sums.lo + sums.hi)


def _alpha(sd, sr, scheme):
    if scheme == "pypower":
        return sd.w_wfkp / sr.w_wfkp
    if scheme == "nbodykit":
        return sd.w / sr.w
    raise ValueError("alpha_scheme must be either 'pypower' or 'nbodykit'.")


# ================================================================== fields
class SurveyField:
    """A painted survey field as the reference holds it: re + i im (im None when
    the paint is not interlaced), n^3 cells of the given precision."""

    def __init__(self, re, im, n, boxsize, sampler, interlaced, precision, boxcenter):
        self.re, self.im = re, im
        self.n = n
        self.boxsize = float(boxsize)
        self.sampler = sampler
        self.window = _lib.WINDOW[sampler]
        self.interlaced = interlaced
        self.precision = precision
        self.code = engine.PRECISION[precision][0]
        self.boxcenter = np.asarray(boxcenter, dtype=np.float64)


def paint_field(items, n, boxsize, sampler, interlaced, boxcenter, precision):
    """pm_painter (mesh_generator.py:172-224) of one or more catalogs into one field.

    ``items``: [(catalog, weights, mass_scale), ...]; the field is
    sum_i mass_scale_i * paint(catalog_i, weights_i) (paint is linear), painted at
    Position - boxcenter.  Interlaced: both meshes, R2C, the split into the
    Hermitian and -i anti-Hermitian parts in place, one batched C2R."""
    ctx = _lib.Context.get()
    code, rdt, cdt = engine.PRECISION[precision]
    dev = _device()
    nb = 2 if interlaced else 1
    mesh = torch.empty((nb, n, n, n), dtype=rdt, device=dev)
    window = _lib.WINDOW[sampler]
    for idx, (cat, w, s) in enumerate(items):
        ctx.paint_ex(code, cat.pos, w, n, float(boxsize), window, boxcenter, s, idx > 0, mesh[0],
                     mesh[1] if interlaced else None)
    if not interlaced:
        return SurveyField(mesh[0], None, n, boxsize, sampler, interlaced, precision, boxcenter)
    spec = torch.empty((2, n, n, n // 2 + 1), dtype=cdt, device=dev)
    ctx.r2c(code, n, 2, mesh, spec)
    ctx.interlace_split(code, n, float(boxsize), spec[0], spec[1], 1.0, False, spec[0], spec[1])
    ctx.c2r(code, n, 2, spec, mesh)
    del spec
    return SurveyField(mesh[0], mesh[1], n, boxsize, sampler, interlaced, precision, boxcenter)


def to_precision(field, precision):
    """The field rounded to ``precision`` once it is formed: the FKP and N fields
    are painted, combined and interlace-split in FP64 (D - alpha R cancels to a
    few per cent of D, which FP32 accumulation would not resolve) and only the
    finished field is held in FP32 for the estimator stages."""
    if precision == field.precision:
        return field
    rdt = engine.PRECISION[precision][1]
    im = None if field.im is None else field.im.to(rdt)
    return SurveyField(field.re.to(rdt), im, field.n, field.boxsize, field.sampler, field.interlaced, precision,
                       field.boxcenter)


def combine(a, X, b, Y):
    """a X + b Y (the x-space field arithmetic of mg:449-454, :666-668)."""
    ctx = _lib.Context.get()
    ncell = X.n ** 3
    re = torch.empty_like(X.re)
    ctx.field_axpby(X.code, ncell, a, X.re, b, Y.re, re)
    im = None
    if X.im is not None or Y.im is not None:
        im = torch.empty_like(X.re)
        if X.im is not None and Y.im is not None:
            ctx.field_axpby(X.code, ncell, a, X.im, b, Y.im, im)
        elif X.im is not None:
            ctx.field_axpby(X.code, ncell, a, X.im, 0.0, None, im)
        else:
            ctx.field_axpby(X.code, ncell, b, Y.im, 0.0, None, im)
    return SurveyField(re, im, X.n, X.boxsize, X.sampler, X.interlaced, X.precision, X.boxcenter)


def product_sum(fields):
    """sum_x prod_j field_j (complex), e.g. np.sum(D * R) of mg:503-519, :829-990."""
    ctx = _lib.Context.get()
    f0 = fields[0]
    out = torch.empty(2, dtype=torch.float64, device=f0.re.device)
    ctx.field_product_sum(f0.code, f0.n ** 3, [f.re for f in fields], [f.im for f in fields], out)
    v = out.cpu().numpy()
    return complex(v[0], v[1])


def forward(field, comp, scale):
    """r2c(field) * compensation * scale as a half spectrum (in-band modes: the
    imaginary residue only lives on modes with a Nyquist component)."""
    ctx = _lib.Context.get()
    _, _, cdt = engine.PRECISION[field.precision]
    n = field.n
    spec = torch.empty((n, n, n // 2 + 1), dtype=cdt, device=field.re.device)
    ctx.r2c(field.code, n, 1, field.re, spec)
    ctx.forward_finish(field.code, n, field.boxsize, spec, None, float(scale), comp, field.window, float("nan"))
    return spec


def harmonic_spectra(field, harm, conj):
    """R2C of Re and Im of field * Y(xhat) (or conj Y): the pair (P, Q) whose
    X = P + i Q is the (unnormalised) FFT of the complex product."""
    ctx = _lib.Context.get()
    _, rdt, cdt = engine.PRECISION[field.precision]
    n = field.n
    need_q = field.im is not None or harm.m != 0
    nb = 2 if need_q else 1
    prod = torch.empty((nb, n, n, n), dtype=rdt, device=field.re.device)
    ctx.xspace_harmonic(field.code, n, field.boxsize, field.boxcenter, field.re, field.im, harm, conj, 1.0,
                        prod[0], prod[1] if need_q else None)
    spec = torch.empty((nb, n, n, n // 2 + 1), dtype=cdt, device=field.re.device)
    ctx.r2c(field.code, n, nb, prod, spec)
    del prod
    return spec[0], (spec[1] if need_q else None)


# ================================================================ pk meshes
def get_mesh_pk_survey(catalogs, correlation_mode, nmesh, geometry, column_names, boxsize, sampler,
                       interlaced, z_range, comp_weight_plan, para_cosmo, normalization_scheme,
                       alpha_scheme="pypower", comm=None, precision="f64"):
    """FKP fields and normalisation of the survey power spectrum (mesh_generator.py:227-538)."""
    n = int(np.array(nmesh)[0])
    L = float(np.array(boxsize)[0])
    dV = np.prod(np.array(boxsize)) / np.prod(np.array(nmesh))

    def read(key, ctype):
        return read_catalog(catalogs[key], column_names, z_range, comp_weight_plan, ctype, para_cosmo,
                            normalization_scheme)

    ra = read("randoms_a", "randoms")
    sr = ParticleSums(ra)
    bc = boxcenter_of(sr)
    da = read("data_a", "data")
    sd = ParticleSums(da)
    if alpha_scheme not in ("pypower", "nbodykit"):
        raise UnboundLocalError("cannot access local variable 'alpha_a' where it is not associated with a value")
    alpha_a = _alpha(sd, sr, alpha_scheme)
    attrs = {"boxcenter": bc, "alpha_a": alpha_a, "I_rand": alpha_a * sr.I_sum, "I_data": sd.I_sum}
    separate = normalization_scheme != "particle"

    def fields(d, r, alpha):
        wd, wr = d.paint_weights(), r.paint_weights()
        if not separate:
            F = paint_field([(d, wd, 1.0 / dV), (r, wr, -alpha / dV)], n, L, sampler, interlaced, bc, "f64")
            return to_precision(F, precision), None, None
        D = paint_field([(d, wd, 1.0 / dV)], n, L, sampler, interlaced, bc, "f64")
        R = paint_field([(r, wr, 1.0 / dV)], n, L, sampler, interlaced, bc, "f64")
        return to_precision(combine(1.0, D, -alpha, R), precision), D, R

    fa, Da, Ra = fields(da, ra, alpha_a)
    fb = fa
    if correlation_mode == "cross":
        db = read("data_b", "data")
        rb = read("randoms_b", "randoms")
        sdb, srb = ParticleSums(db), ParticleSums(rb)
        alpha_b = sdb.w_wfkp / srb.w_wfkp if alpha_scheme == "pypower" else sdb.w / srb.w
        attrs["alpha_b"] = alpha_b
        fb, Db, Rb = fields(db, rb, alpha_b)
    if normalization_scheme == "particle":
        if correlation_mode == "auto":
            attrs["N0"] = (sd.N_sum + alpha_a ** 2 * sr.N_sum) / attrs["I_rand"]
        else:
            raise ValueError("Particle-normalization scheme will not work for cross-correlation!")
    else:
        if correlation_mode == "auto":
            I_mesh = alpha_a * product_sum([Da, Ra]) * np.prod(boxsize) / np.prod(nmesh)
        else:
            I_mesh = 0.5 * np.prod(boxsize) / np.prod(nmesh) * (
                attrs["alpha_b"] * product_sum([Da, Rb]) + alpha_a * product_sum([Db, Ra]))
        I_mesh = np.float64(np.real(I_mesh))
        attrs["I_mesh"] = I_mesh
        attrs["N0"] = (sd.N_sum + alpha_a ** 2 * sr.N_sum) / I_mesh if correlation_mode == "auto" else 0.0
    return attrs, fa, fb


# ====================================================================== pk
_SUPPORTED_HIGH = ([0, 2, 4], [0, 2, 4, 6], [0, 2, 4, 6, 8])


def _high_order_strategy(poles, mode, correlation_mode):
    """get_high_order_strategy (clustering_estimator.py:243-331)."""
    if mode == "default" or correlation_mode != "auto" or poles not in _SUPPORTED_HIGH:
        return None
    high = {p for p in poles if p in (4, 6, 8)}
    if mode == "fast":
        fast = {(0, 2, 4): {4}, (0, 2, 4, 6): {6}, (0, 2, 4, 6, 8): {6, 8}}[tuple(poles)]
        exact = {(0, 2, 4): set(), (0, 2, 4, 6): {4}, (0, 2, 4, 6, 8): {4}}[tuple(poles)]
    else:
        fast, exact = set(high), set(high)
    internal = {4} if fast & {6, 8} else set()
    return {"mode": mode, "fast": fast, "exact": exact | internal, "visible": exact,
            "f2": bool(fast & {4, 6, 8}), "f4": bool(fast & {6, 8})}


def _bins(field, u, v, edges, harm=None, conj_z=False, weight=1.0, sbar=0.0):
    ctx = _lib.Context.get()
    d = torch.empty(2 * (len(edges) - 1), dtype=torch.float64, device=field.re.device)
    ctx.survey_bins(field.code, field.n, field.boxsize, field.window, u, v, sbar, harm, conj_z, weight, edges, d)
    return engine.HostCopy(d)


def _complex_of(hc):
    v = hc.get()
    return v[0::2] + 1j * v[1::2]


def calculate_power_spectrum_survey(stat_attrs, rfield_a, rfield_b, correlation_mode, comm=None, **kwargs):
    """Survey power-spectrum multipoles (clustering_estimator.py:205-563)."""
    poles = stat_attrs["poles"]
    mode = stat_attrs.get("high_order_mode", "default")
    boxsize, nmesh = np.array(stat_attrs["boxsize"]), np.array(stat_attrs["nmesh"])
    k_min, k_max, k_bins = stat_attrs["k_min"], stat_attrs["k_max"], stat_attrs["k_bins"]
    N0 = stat_attrs["N0"]
    I_norm = stat_attrs["I_rand"] if stat_attrs["normalization_scheme"] == "particle" else stat_attrs["I_mesh"]
    k_edge = np.linspace(k_min, k_max, k_bins + 1)
    strat = _high_order_strategy(poles, mode, correlation_mode)
    ctx = _lib.Context.get()
    fa, fb = rfield_a, rfield_b
    n, L = fa.n, fa.boxsize
    V = float(boxsize.prod())
    comp = _lib.COMP_SINC if fa.interlaced else _lib.COMP_SHOTNOISE
    ca = forward(fa, comp, V)
    cb = ca if correlation_mode == "auto" else forward(fb, comp, V)
    counts = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k_edge)))
    opa = ctx.operand(ca)
    opb = ctx.operand(cb)
    pending = {}
    F = {}
    for pole in poles:
        if pole == 0:
            pending[0] = [_bins(fa, opa, opb, k_edge)]
            continue
        store = True
        if pole in (4, 6, 8) and strat is not None:
            store = pole in strat["exact"]
        cache2 = pole == 2 and strat is not None and strat["f2"]
        cache4 = pole == 4 and strat is not None and strat["f4"]
        if not (store or cache2 or cache4):
            continue
        scale = (4.0 * np.pi * V / (2 * pole + 1)) / float(n) ** 3
        if cache2 or cache4:
            F[pole] = torch.zeros_like(ca)
        parts = []
        for m in range(pole + 1):
            h = angular.harmonic(pole, m, racah=False)
            P, Q = harmonic_spectra(fb, h, conj=m > 0)
            x = ctx.operand(P, Q, scale, comp)
            w = 1.0 if m == 0 else 2.0
            if store:
                parts.append(_bins(fa, opa, x, k_edge, h, True, w))
            if pole in F:
                ctx.hermitian_accumulate(fa.code, n, L, fa.window, x, h, w, F[pole])
            del P, Q
        if store:
            pending[pole] = parts
    c = counts.get()
    k_num = c[0].copy()
    k_eff = c[1] / c[0]
    results = {"k_eff": k_eff, "k_num": k_num, "I_norm": I_norm}
    for pole in poles:
        if pole not in pending:
            continue
        total = sum(_complex_of(h) for h in pending[pole])
        if pole == 0 and correlation_mode == "auto":
            total = np.real(total)
        res = total / k_num
        res *= (2 * pole + 1) / I_norm
        if pole == 0:
            res -= N0
        else:
            res = np.imag(res) if pole & 1 else np.real(res)
        results[f"P{pole}"] = res
    if strat is not None and strat["fast"]:
        op2 = ctx.operand(F[2])
        if 4 in strat["fast"]:
            P22 = np.real(_complex_of(_bins(fa, op2, op2, k_edge))) / k_num
            P22 *= 9 / I_norm
            P22 -= N0 * 9 / 5
            results["P4b"] = np.real(35 / 18 * P22 - results["P2"] - 7 / 2 * results["P0"])
        if strat["fast"] & {6, 8}:
            op4 = ctx.operand(F[4])
            s42 = _complex_of(_bins(fa, op4, op2, k_edge))
            if 6 in strat["fast"]:
                P42 = s42 / k_num
                P42 *= 13 / I_norm
                results["P6b"] = np.real(11 / 5 * P42 - 52 / 63 * results["P4"] - 286 / 175 * results["P2"])
            if 8 in strat["fast"]:
                P42 = s42 / k_num
                P42 *= 13 / I_norm
                P44 = np.real(_complex_of(_bins(fa, op4, op4, k_edge))) / k_num
                P44 *= 17 / I_norm
                P44 -= N0 * 17 / 9
                results["P8b"] = np.real(1287 / 490 * P44 - 374 / 245 * P42 - 3553 / 15435 * results["P4"]
                                         - 1326 / 8575 * results["P2"] - 2431 / 490 * results["P0"])
        if strat["mode"] == "fast":
            for p in strat["fast"]:
                results.pop(f"P{p}", None)
    return results


# ================================================================ bk meshes
def get_mesh_bk_survey(catalogs, correlation_mode, tracer_type, angu_config, nmesh, geometry, column_names,
                       boxsize, sampler, interlaced, z_range, comp_weight_plan, para_cosmo, comm=None,
                       normalization_scheme="particle", alpha_scheme="pypower", precision="f64"):
    """FKP fields and I_norm of the survey bispectrum (mesh_generator.py:541-1004)."""
    assert geometry == "survey-like", "get_mesh_bk_survey only supports survey-like geometry."
    assert correlation_mode in ["auto", "cross"], "correlation_mode must be 'auto' or 'cross'."
    assert tracer_type in ["aaa", "aab", "abb", "abc"], \
        "tracer_type must be one of 'aaa', 'aab', 'abb', 'abc'."
    assert normalization_scheme in ["particle", "mesh", "mixed-mesh"], \
        "normalization_scheme must be one of 'particle', 'mesh', 'mixed-mesh'."
    if correlation_mode == "auto":
        assert tracer_type == "aaa", "For auto-correlation, tracer_type must be 'aaa'."
    n = int(np.array(nmesh)[0])
    L = float(np.array(boxsize)[0])
    dV = np.prod(np.array(boxsize)) / np.prod(np.array(nmesh))
    L_ = angu_config[2]

    def read(key, ctype):
        return read_catalog(catalogs[key], column_names, z_range, comp_weight_plan, ctype, para_cosmo,
                            normalization_scheme)

    bc = boxcenter_of(ParticleSums(read("randoms_a", "randoms")))
    attrs = {"normalization_scheme": normalization_scheme, "boxcenter": bc}
    keep = {t: {"D": False, "R": False} for t in "abc"}
    if normalization_scheme == "mesh":
        keep["a"]["R"] = True
    elif normalization_scheme == "mixed-mesh":
        if correlation_mode == "auto":
            keep["a"]["D"] = True
        elif tracer_type == "abc":
            keep["a"]["R"] = keep["b"]["R"] = keep["c"]["R"] = True
        elif tracer_type == "aab":
            keep["a"]["D"] = keep["a"]["R"] = keep["b"]["R"] = True
        elif tracer_type == "abb":
            keep["a"]["R"] = keep["b"]["R"] = keep["b"]["D"] = True
    fields, cache = {}, {}

    def prep(label):
        r = read(f"randoms_{label}", "randoms")
        d = read(f"data_{label}", "data")
        auto = correlation_mode == "auto"
        sd = ParticleSums(d, L_ if auto else None)
        sr = ParticleSums(r, L_ if auto else None)
        alpha = _alpha(sd, sr, alpha_scheme)
        attrs[f"alpha_{label}"] = alpha
        attrs[f"I_33_{label}"] = sr.I33 * alpha
        attrs[f"S_LM_{label}"] = (sd.S_LM - alpha ** 3 * sr.S_LM) if auto else 0.0
        wd, wr = d.paint_weights(), r.paint_weights()
        if not (keep[label]["D"] or keep[label]["R"]):
            F = paint_field([(d, wd, 1.0 / dV), (r, wr, -alpha / dV)], n, L, sampler, interlaced, bc, "f64")
        else:
            D = paint_field([(d, wd, 1.0 / dV)], n, L, sampler, interlaced, bc, "f64")
            R = paint_field([(r, wr, alpha / dV)], n, L, sampler, interlaced, bc, "f64")
            F = combine(1.0, D, -1.0, R)
            cache[label] = (D if keep[label]["D"] else None, R if keep[label]["R"] else None)
        fields[label] = to_precision(F, precision)

    prep("a")
    if correlation_mode == "cross":
        prep("b")
        if tracer_type == "abc":
            prep("c")
    if normalization_scheme == "particle":
        assert correlation_mode == "auto", "Particle-normalization scheme is only applicable for auto-correlation."
        attrs["I_norm"] = attrs["I_33_a"]
    elif normalization_scheme == "mesh":
        assert correlation_mode == "auto", "Mesh-normalization scheme is only applicable for auto-correlation."
        R = cache["a"][1]
        attrs["I_norm"] = dV * product_sum([R, R, R])
    elif correlation_mode == "auto":
        D = cache["a"][0]
        d = read("data_a", "data")
        r = read("randoms_a", "randoms")
        ro, re_ = r.take(slice(1, None, 2)), r.take(slice(0, None, 2))
        if alpha_scheme not in ("pypower", "nbodykit"):
            raise ValueError("alpha_scheme must be either 'pypower' or 'nbodykit'.")
        sd, so, se = ParticleSums(d), ParticleSums(ro), ParticleSums(re_)
        a_odd, a_even = _alpha(sd, so, alpha_scheme), _alpha(sd, se, alpha_scheme)
        Ro = paint_field([(ro, ro.paint_weights(), a_odd / dV)], n, L, sampler, interlaced, bc, "f64")
        Re = paint_field([(re_, re_.paint_weights(), a_even / dV)], n, L, sampler, interlaced, bc, "f64")
        attrs["I_norm"] = dV * product_sum([D, Ro, Re])
    else:
        if tracer_type == "abc":
            trio = [cache["a"][1], cache["b"][1], cache["c"][1]]
        elif tracer_type == "aab":
            trio = [cache["a"][0], cache["a"][1], cache["b"][1]]
        else:
            trio = [cache["a"][1], cache["b"][1], cache["b"][0]]
        attrs["I_norm"] = dV * product_sum(trio)
    cache.clear()
    return attrs, fields["a"], fields.get("b"), fields.get("c")


def get_N_field(catalogs, tracer_flag, alpha, nmesh, geometry, column_names, boxsize, sampler, interlaced,
                z_range, comp_weight_plan, para_cosmo, boxcenter, comm=None, normalization_scheme="particle",
                precision="f64"):
    """(D_{w^2} + alpha^2 R_{w^2}) / dV (mesh_generator.py:1007-1128)."""
    assert geometry == "survey-like", "get_N_field currently supports survey-like geometry only."
    assert tracer_flag in ["a", "b", "c"], "tracer_flag must be one of 'a', 'b', or 'c'."
    n = int(np.array(nmesh)[0])
    L = float(np.array(boxsize)[0])
    dV = np.prod(np.array(boxsize)) / np.prod(np.array(nmesh))
    r = read_catalog(catalogs[f"randoms_{tracer_flag}"], column_names, z_range, comp_weight_plan, "randoms",
                     para_cosmo, normalization_scheme)
    d = read_catalog(catalogs[f"data_{tracer_flag}"], column_names, z_range, comp_weight_plan, "data",
                     para_cosmo, normalization_scheme)
    N = paint_field([(d, d.paint_weights(2), 1.0 / dV), (r, r.paint_weights(2), alpha ** 2 / dV)],
                    n, L, sampler, interlaced, boxcenter, "f64")
    return to_precision(N, precision)


# ====================================================================== bk
def _g_lm(field3, L_, M, band):
    """G_LM = c2r(comp r2c(rfield3 Y_LM(xhat))) (ce:1697-1713), band-limited to the
    |k| < 2 k_max its triple sums can see; returns (Re G, Im G or None)."""
    ctx = _lib.Context.get()
    n = field3.n
    P, Q = harmonic_spectra(field3, angular.harmonic(L_, M, True), False)
    out = []
    for s in (P, Q):
        if s is None:
            out.append(None)
            continue
        ctx.forward_finish(field3.code, n, field3.boxsize, s, None, 1.0, _lib.COMP_SINC, field3.window,
                           float("nan"), band)
        f = torch.empty(n * n * n, dtype=engine.PRECISION[field3.precision][1], device=s.device)
        ctx.c2r(field3.code, n, 1, s, f)
        out.append(f)
    return out[0], out[1]


def _signal_spec(l1, l2, m1, m2, same12, tracer_type):
    leg1 = (l1, m1, 0, False)
    if same12 and l1 == l2 and m1 == m2:
        return engine.PairSpec(leg1, "eq")
    if same12 and l1 == l2 and m1 == -m2:
        return engine.PairSpec(leg1, "conj", sign=(-1.0) ** (m1 + l1))
    return engine.PairSpec(leg1, "leg", (l2, m2, 0 if tracer_type in ("aaa", "aab") else 1, False))


def _s3_spec(l1, l2, m1, m2):
    leg1 = (l1, m1, 2, True)
    if l1 == l2 and m1 == m2:
        return engine.PairSpec(leg1, "eq")
    if l1 == l2 and m1 == -m2:
        return engine.PairSpec(leg1, "conj", sign=(-1.0) ** (m1 + l1))
    return engine.PairSpec(leg1, "leg", (l2, m2, 2, True))


def _complex_pairs(groups_by_key, sf, k_bins, diagonal, bs):
    """pair_sums with complex weight fields: {key: (Gr, Gi, spec)} ->
    {key: deferred (S_r, S_i)} where S = S_r + i S_i."""
    keys = list(groups_by_key)
    groups, index = [], []
    for k in keys:
        Gr, Gi, ps = groups_by_key[k]
        index.append((k, len(groups), None if Gi is None else len(groups) + 1))
        groups.append((Gr, [ps]))
        if Gi is not None:
            groups.append((Gi, [ps]))
    outs = engine.pair_sums(groups, sf, k_bins, diagonal, bs)
    return {k: (outs[ir], None if ii is None else outs[ii]) for (k, ir, ii) in index}


def _resolve(pair):
    r, i = pair
    S = r.result()[0]
    if i is not None:
        S = S + 1j * i.result()[0]
    return S


def _symmetric_fill(sub, eq, cj):
    k = sub.shape[0]
    for i in range(k):
        for j in range(i + 1, k):
            if eq:
                sub[j, i] = sub[i, j]
            elif cj:
                sub[j, i] = np.conj(sub[i, j])
    return sub


def calculate_bk_sugi_survey(rfield_a, rfield_b, rfield_c, correlation_mode, stat_attrs, comm=None, **kwargs):
    """Survey Sugiyama bispectrum with shot noise (clustering_estimator.py:1558-3101)."""
    data_vector_mode = stat_attrs.get("data_vector_mode", "diagonal")
    shotnoise_mode = stat_attrs.get("shotnoise_mode", "ana")
    block_size = stat_attrs.get("block_size", 1 if data_vector_mode == "diagonal" else "full")
    l1, l2, L_ = stat_attrs["angu_config"]
    boxsize, nmesh = np.array(stat_attrs["boxsize"]), np.array(stat_attrs["nmesh"])
    k_min, k_max, k_bins = stat_attrs["k_min"], stat_attrs["k_max"], stat_attrs["k_bins"]
    tracer_type = stat_attrs["tracer_type"]
    I_norm = stat_attrs["I_norm"]
    vol_per_cell = boxsize.prod() / nmesh.prod()
    N_ells = (2 * l1 + 1) * (2 * l2 + 1) * (2 * L_ + 1)
    H_ells = angular.wigner3j(l1, l2, L_, 0, 0, 0)
    cfgs, tj = angular.magnetic_configs_survey(l1, l2, L_)
    k_edge = np.linspace(k_min, k_max, k_bins + 1)
    if data_vector_mode not in ("diagonal", "full"):
        raise ValueError("data_vector_mode must be either 'diagonal' or 'full'.")
    diagonal = data_vector_mode == "diagonal"
    fa = rfield_a
    n, L = fa.n, fa.boxsize
    V = float(boxsize.prod())
    precision = fa.precision
    ctx = _lib.Context.get()
    band = 2.0 * k_max

    ca = forward(fa, _lib.COMP_SINC, V)
    cb = ca if correlation_mode == "auto" else forward(rfield_b, _lib.COMP_SINC, V)
    counts = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k_edge)))
    k3_edge = np.linspace(2 * k_min, 2 * k_max, k_bins * 2 + 1)[:-1]
    k3_center = 0.5 * (k3_edge[1:] + k3_edge[:-1])
    k3_bins = len(k3_center)
    counts3 = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k3_edge)))
    field3 = fa if correlation_mode == "auto" else (rfield_c if tracer_type == "abc" else rfield_b)

    # ---- signal: configurations in order, G_LM recomputed when M changes (ce:1720-1945)
    same12 = correlation_mode == "auto" or tracer_type == "aab"
    idx = {c: i for i, c in enumerate(cfgs)}
    plan, done = [], set()
    for ss, (m1, m2, M) in enumerate(cfgs):
        if (m1, m2, M) in done:
            continue
        swap = (m2, m1, M)
        add_swap = same12 and l1 == l2 and swap in idx and swap != (m1, m2, M) and swap not in done
        plan.append((ss, m1, m2, M, add_swap))
        if add_swap:
            done.add(swap)
        done.add((m1, m2, M))
    specs = {ss: _signal_spec(l1, l2, m1, m2, same12, tracer_type) for (ss, m1, m2, M, _) in plan}
    bs, capacity = _plan_signal_blocks(list(specs.values()), k_bins, n, precision, block_size, diagonal)
    sf = engine.ShellFields(n, L, k_edge, precision, ca, cb if cb is not ca else None, capacity=capacity)
    sig = {}
    Gs = {}
    for M in dict.fromkeys(M for (_, _, _, M, _) in plan):
        Gr, Gi = _g_lm(field3, L_, M, band)
        group = {ss: (Gr, Gi, specs[ss]) for (ss, _, _, MM, _) in plan if MM == M}
        sig.update(_complex_pairs(group, sf, k_bins, diagonal, bs))
        Gs[M] = (Gr, Gi)
    del sf

    # ---- shot noise fields (ce:2070-2186)
    rshot = Nshot = S_LM = None
    nfield_kw = dict(nmesh=stat_attrs["nmesh"], geometry="survey-like", column_names=stat_attrs["column_names"],
                     boxsize=stat_attrs["boxsize"], sampler=stat_attrs["sampler"],
                     interlaced=stat_attrs["interlaced"], z_range=stat_attrs["z_range"],
                     comp_weight_plan=stat_attrs["comp_weight_plan"], para_cosmo=stat_attrs["cosmology"],
                     boxcenter=stat_attrs["boxcenter"],
                     normalization_scheme=stat_attrs.get("normalization_scheme", "particle"), precision=precision)
    catalogs = kwargs.get("catalogs", None)
    if catalogs is None:
        raise ValueError("catalogs must be provided to calculate_bk_sugi_survey for N_field construction.")
    if tracer_type == "aab":
        rshot, cshot = rfield_b, cb
        Nshot = get_N_field(catalogs, "a", stat_attrs["alpha_a"], **nfield_kw)
        S_LM = stat_attrs.get("S_LM_a", None)
    elif tracer_type == "abb":
        rshot, cshot = rfield_a, ca
        Nshot = get_N_field(catalogs, "b", stat_attrs["alpha_b"], **nfield_kw)
        S_LM = stat_attrs.get("S_LM_b", None)
    elif tracer_type != "abc":
        rshot, cshot = rfield_a, ca
        Nshot = get_N_field(catalogs, "a", stat_attrs["alpha_a"], **nfield_kw)
        S_LM = stat_attrs.get("S_LM_a", None)
    sbar_on = correlation_mode == "auto" and tracer_type == "aaa"
    S_arr = None
    if sbar_on:
        if S_LM is None:
            S_arr = np.zeros(L_ + 1, dtype="complex128")
        elif np.isscalar(S_LM):
            S_arr = np.zeros(L_ + 1, dtype="complex128")
            S_arr[0] = S_LM
        else:
            S_arr = np.asarray(S_LM, dtype="complex128")
    scale_nv = V / float(n) ** 3

    s1_parts, q_parts = [], []
    s3fft = None
    if tracer_type != "abc":
        if tracer_type in ("aaa", "abb") and l1 == L_ and l2 == 0:
            opd = ctx.operand(cshot)
            for M in range(L_ + 1):
                h = angular.harmonic(L_, M, True)
                P, Q = harmonic_spectra(Nshot, h, False)
                x = ctx.operand(P, Q, scale_nv, _lib.COMP_SINC)
                sb = S_arr[M] if sbar_on else 0.0
                s1_parts.append(_bins(fa, opd, x, k_edge, h, False, 0.5 if M == 0 else 1.0, sb))
                del P, Q
        if tracer_type != "abb":
            cN00 = forward(Nshot, _lib.COMP_SINC, V)
            opn = ctx.operand(cN00)
            if shotnoise_mode in ("ana", "both"):
                for M in range(L_ + 1):
                    h = angular.harmonic(L_, M, True)
                    P, Q = harmonic_spectra(rshot, h, True)
                    x = ctx.operand(P, Q, scale_nv, _lib.COMP_SINC)
                    sb = S_arr[M] if sbar_on else 0.0
                    q_parts.append(_bins(fa, x, opn, k3_edge, h, False, 0.5 if M == 0 else 1.0, sb))
                    del P, Q
            if shotnoise_mode in ("fft", "both"):
                s3fft = _s3_fft_sums(rshot, opn, cfgs, l1, l2, L_, S_arr, k_edge, k_bins, diagonal, block_size,
                                     band, scale_nv)
            del cN00
    del Nshot

    # ---- host algebra
    c = counts.get()
    k_num, k_eff = c[0].copy(), c[1] / c[0]
    c3 = counts3.get()
    k_num_k3, k3_eff = c3[0].copy(), c3[1] / c3[0]
    shape = (k_bins,) if diagonal else (k_bins, k_bins)

    total = np.zeros(shape, dtype="complex128")
    for (ss, m1, m2, M, add_swap) in plan:
        S = _resolve(sig[ss])
        sub = tj[ss] * S
        ps = specs[ss]
        if not diagonal and ps.mode in ("eq", "conj"):
            sub = _symmetric_fill(sub, ps.mode == "eq", ps.mode == "conj")
        if add_swap:
            sub = 2.0 * sub if diagonal else sub + sub.T
        total += sub if (m1, m2, M) == (0, 0, 0) else 2 * np.real(sub)

    SN0 = 0.0 + 0.0j
    SN1 = np.zeros(shape, dtype="complex128")
    SN2 = np.zeros(shape, dtype="complex128")
    SN3 = np.zeros(shape, dtype="complex128")
    SN3_fft = None
    if tracer_type != "abc":
        if tracer_type == "aaa" and (l1 == 0 and l2 == 0 and L_ == 0):
            S_a = stat_attrs.get("S_LM_a", 0.0)
            SN0 = S_a[0] if isinstance(S_a, np.ndarray) else S_a
        if s1_parts:
            tot = 2.0 * np.real(sum(_complex_of(h) for h in s1_parts))
            vec = np.zeros(k_bins, dtype="complex128")
            ok = k_num > 0
            vec[ok] = (2 * L_ + 1) * tot[ok] / k_num[ok]
            if diagonal:
                SN1 = vec
            else:
                for i in range(k_bins):
                    SN1[i, :] = vec[i]
            if tracer_type == "aaa" and (l1 == 0 and l2 == 0 and L_ == 0):
                if diagonal:
                    SN2 = vec.copy()
                else:
                    for i in range(k_bins):
                        SN2[:, i] = vec[i]
        if tracer_type != "abb":
            if q_parts:
                Q_like = (2.0 * np.real(sum(_complex_of(h) for h in q_parts))).astype("complex128")
                q = angular.q_ells_matrix(k_eff, l1, l2, L_, k3_eff)
                SN3 = angular.s3_analytic(Q_like, k_num_k3, k_edge, k3_center, q, diagonal) * (H_ells * N_ells)
            if s3fft is not None:
                s3 = _s3_fft_assemble(s3fft, cfgs, tj, l1, l2, k_num, k_bins, diagonal)
                s3 *= H_ells * N_ells
                s3 *= 1 / nmesh.prod()
                if shotnoise_mode == "fft":
                    SN3 = s3
                else:
                    SN3_fft = s3
        elif shotnoise_mode == "both":
            SN3_fft = np.zeros(shape, dtype="complex128")

    total *= N_ells * H_ells / I_norm
    total *= 1.0 / (np.outer(k_num, k_num) if not diagonal else k_num ** 2)
    total *= vol_per_cell
    shot = (SN0 + SN1 + SN2 + SN3) / I_norm
    sn_terms = {"SN0": SN0 / I_norm, "SN1": SN1 / I_norm, "SN2": SN2 / I_norm, "SN3": SN3 / I_norm}
    if shotnoise_mode == "both":
        # the reference divides None by I_norm here for tracer "abc" (TypeError)
        sn_terms["SN3_FFT"] = SN3_fft / I_norm
    return {"B_sugi": total - shot, "Bk_raw": total, "SN_terms": sn_terms, "Shot_noise": shot,
            "I_norm": I_norm, "k_eff": k_eff, "nmodes": k_num}


def _plan_signal_blocks(specs, k_bins, n, precision, block_size, diagonal):
    from .clustering_estimator import _plan_blocks

    return _plan_blocks(specs, k_bins, n, precision, block_size, diagonal)


def _s3_fft_sums(rshot, opn, cfgs, l1, l2, L_, S_arr, k_edge, k_bins, diagonal, block_size, band, scale_nv):
    """FFT S3 (ce:2403-2781): per M the complex source c2r(delta_LM conj N00 -
    Sbar W) split into real fields, contracted with the data-independent shells
    c2r(conj Y mask) of every configuration."""
    ctx = _lib.Context.get()
    n = rshot.n
    _, rdt, cdt = engine.PRECISION[rshot.precision]
    idx = {c: i for i, c in enumerate(cfgs)}
    plan, done = [], set()
    for ss, (m1, m2, M) in enumerate(cfgs):
        if (m1, m2, M) in done:
            continue
        swap = (m2, m1, M)
        add_swap = l1 == l2 and swap in idx and swap != (m1, m2, M) and swap not in done
        plan.append((ss, m1, m2, M, add_swap))
        if add_swap:
            done.add(swap)
        done.add((m1, m2, M))
    specs = {ss: _s3_spec(l1, l2, m1, m2) for (ss, m1, m2, M, _) in plan}
    bs, capacity = _plan_signal_blocks(list(specs.values()), k_bins, n, rshot.precision, block_size, diagonal)
    sf = engine.ShellFields(n, rshot.boxsize, k_edge, rshot.precision, None, None, capacity=capacity)

    def s_val(Mi):
        if S_arr is None:
            return 0.0 + 0.0j
        return S_arr[Mi] if Mi >= 0 else ((-1) ** Mi) * np.conj(S_arr[-Mi])

    sums, origin = {}, {}
    for M in dict.fromkeys(M for (_, _, _, M, _) in plan):
        P, Q = harmonic_spectra(rshot, angular.harmonic(L_, M, True), True)
        x = ctx.operand(P, Q, scale_nv, _lib.COMP_SINC)
        src = torch.empty((2, n, n, n // 2 + 1), dtype=cdt, device=P.device)
        ctx.survey_source(rshot.code, n, rshot.boxsize, rshot.window, x, opn, s_val(M), band, src[0], src[1])
        if rshot.precision == "f32":
            # x = 0 cell added in FP64 (engine.origin_correction)
            d0 = torch.empty(2, dtype=torch.float64, device=src.device)
            ctx.survey_bins(rshot.code, n, rshot.boxsize, rshot.window, x, opn, s_val(M), None, False, 1.0,
                            [0.0, band], d0)
            origin[M] = engine.HostCopy(d0)
        del P, Q, x
        fld = torch.empty((2, n * n * n), dtype=rdt, device=src.device)
        ctx.c2r(rshot.code, n, 2, src, fld)
        del src
        if rshot.precision == "f32":
            fld[:, 0:1].zero_()
        group = {ss: (fld[0], fld[1], specs[ss]) for (ss, _, _, MM, _) in plan if MM == M}
        sums.update(_complex_pairs(group, sf, k_bins, diagonal, bs))
    shell_origin = None
    if origin:
        legs = [ps.leg1 for ps in specs.values()] + [ps.leg2 for ps in specs.values() if ps.mode == "leg"]
        shell_origin = engine.unit_shell_origin(n, rshot.boxsize, k_edge, rshot.precision, legs)
    return plan, specs, sums, origin, shell_origin


def _s3_fft_assemble(s3fft, cfgs, tj, l1, l2, k_num, k_bins, diagonal):
    plan, specs, sums, origin, shell_origin = s3fft
    out = np.zeros((k_bins,) if diagonal else (k_bins, k_bins), dtype="complex128")
    for (ss, m1, m2, M, add_swap) in plan:
        S = _resolve(sums[ss])
        if origin:
            v0 = origin[M].get()
            S = S + engine.origin_correction(specs[ss], shell_origin, complex(v0[0], v0[1]), k_bins, diagonal)
        if diagonal:
            sub = np.zeros(k_bins, dtype="complex128")
            ok = k_num > 0
            sub[ok] = tj[ss] * S[ok] / (k_num[ok] ** 2)
        else:
            sub = np.zeros((k_bins, k_bins), dtype="complex128")
            ok = np.outer(k_num > 0, k_num > 0)
            with np.errstate(divide="ignore", invalid="ignore"):
                sub[ok] = (tj[ss] * S / np.outer(k_num, k_num))[ok]
            ps = specs[ss]
            if ps.mode in ("eq", "conj"):
                sub = _symmetric_fill(sub, ps.mode == "eq", ps.mode == "conj")
        if add_swap:
            sub = 2.0 * sub if diagonal else sub + sub.T
        out += sub if (m1, m2, M) == (0, 0, 0) else 2.0 * np.real(sub)
    return out
