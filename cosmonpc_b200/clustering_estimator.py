"""Box-geometry estimators on the device (drop-in for the reference's
``calculate_power_spectrum_box`` and ``calculate_bk_sugi_box``).

Inputs are :class:`engine.PaintedMesh` objects (the painted "rfields"); outputs
are the same result dictionaries, keys and dtypes as the reference
(src/cosmonpc/clustering_estimator.py:566-746 and :749-1555).  Host code here
only does O(k_bins^2) scalar algebra in FP64; every per-mode and per-cell sum
runs on the GPU.
"""
from __future__ import annotations

import logging

import numpy as np
import torch

from . import _lib, angular, engine


def _precision(stat_attrs, kwargs):
    p = kwargs.get("precision", stat_attrs.get("precision", "f64"))
    if p not in engine.PRECISION:
        raise ValueError("precision must be 'f64' or 'f32'")
    return p


# ===================================================================== pk
def calculate_power_spectrum_box(rfield_a, rfield_b, correlation_mode, stat_attrs, comm=None, **kwargs):
    """Power-spectrum multipoles in a periodic box (clustering_estimator.py:566-746)."""
    poles = stat_attrs["poles"]
    boxsize, nmesh = np.array(stat_attrs["boxsize"]), np.array(stat_attrs["nmesh"])
    k_min, k_max, k_bins = stat_attrs["k_min"], stat_attrs["k_max"], stat_attrs["k_bins"]
    sampler, interlaced = stat_attrs["sampler"], stat_attrs["interlaced"]
    rsd = np.array(stat_attrs["rsd"], dtype=np.float64)
    P_shot = 1.0 / stat_attrs["NZ_a"] if correlation_mode == "auto" else 0.0
    NZ_a = stat_attrs["NZ_a"]
    NZ_b = stat_attrs["NZ_b"] if correlation_mode == "cross" else None
    n = int(nmesh[0])
    L = float(boxsize[0])

    k_edge = np.linspace(k_min, k_max, k_bins + 1)
    comp = _lib.COMP_SINC if interlaced else _lib.COMP_SHOTNOISE
    # r2c + compensation, zero mode cleared (ce:599-636)
    ca = engine.finish_delta(rfield_a, 1.0, comp, 0.0)
    cb = engine.finish_delta(rfield_b, 1.0, comp, 0.0) if correlation_mode == "cross" else ca
    prec = rfield_a.precision
    code = engine.PRECISION[prec][0]

    counts = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k_edge)))
    even = [p for p in poles if not p & 1]
    dsum = None
    if even:
        ctx = _lib.Context.get()
        dsum = torch.empty((len(even), k_bins), dtype=torch.float64, device=ca.device)
        ctx.pk_bins(code, n, L, ca, cb, k_edge, even, rsd, dsum)
        dsum = engine.HostCopy(dsum)
    def finalize(NZ_a=NZ_a):
        """``NZ_a``: the number density of a catalog whose device work ran with
        another count (a padded CUDA-graph capture); only host algebra uses it."""
        P_shot = 1.0 / NZ_a if correlation_mode == "auto" else 0.0
        return _pk_box_results(counts, dsum, poles, even, k_bins, correlation_mode, boxsize, nmesh, NZ_a, NZ_b,
                               P_shot)

    return finalize if kwargs.get("deferred") else finalize()


def _pk_box_results(counts, dsum, poles, even, k_bins, correlation_mode, boxsize, nmesh, NZ_a, NZ_b, P_shot):
    c = counts.get()
    sums = dsum.get() if dsum is not None else None
    k_num = c[0].copy()
    k_eff = c[1] / c[0]
    results = {"k_eff": k_eff, "k_num": k_num}
    for pole in poles:
        if pole & 1:
            res = np.zeros(k_bins).astype("float128")
        else:
            res = sums[even.index(pole)] / k_num
            if correlation_mode == "auto":
                res *= boxsize.prod() ** (-1) * (nmesh.prod() ** 2) / NZ_a ** 2
            else:
                res *= boxsize.prod() ** (-1) * nmesh.prod() ** 2 / (NZ_a * NZ_b)
            if pole == 0:
                res -= P_shot
            else:
                res *= 2 * pole + 1
        results.update({"P%d" % pole: res, "P_shot": P_shot})
    return results


# ================================================================ bk_sugi
def _legs_for_signal(l1, l2, m1, m2, correlation_mode, tracer_type):
    """Which fields feed the two shell legs (clustering_estimator.py:898-970)."""
    leg1 = (l1, m1, 0, False)
    same_tracer = correlation_mode == "auto" or tracer_type == "aab"
    if same_tracer and l1 == l2 and m1 == m2:
        return engine.PairSpec(leg1, "eq")
    if same_tracer and l1 == l2 and m1 == -m2:
        return engine.PairSpec(leg1, "conj", sign=(-1.0) ** (m1 + l1))
    src2 = 0 if tracer_type in ("aaa", "aab") else 1
    return engine.PairSpec(leg1, "leg", (l2, m2, src2, False))


def _legs_for_s3fft(l1, l2, m1, m2):
    """Shell legs of the FFT S3 term: conj(Y) on a unit spectrum (ce:1215-1219)."""
    leg1 = (l1, m1, 2, True)
    if l1 == l2 and m1 == m2:
        return engine.PairSpec(leg1, "eq")
    if l1 == l2 and m1 == -m2:
        return engine.PairSpec(leg1, "conj", sign=(-1.0) ** (m1 + l1))
    return engine.PairSpec(leg1, "leg", (l2, m2, 2, True))


def _plan_blocks(specs, k_bins, n, precision, requested, diagonal, free_bytes=None):
    """Bin block size and shell-field capacity for one pair_sums call.

    ``requested`` is the reference's block_size (ce:867-879): "full"/None means all
    bins at once.  The block is the largest one whose fields fit the HBM budget
    (autotune: a block of all bins computes each field once; smaller blocks
    recompute them), capped by the request.
    """
    if diagonal or requested == "full" or requested is None:
        bs = k_bins
    elif isinstance(requested, (int, np.integer)) and 1 <= requested <= k_bins:
        bs = int(requested)
    else:
        raise ValueError("For full mode, block_size must be 1, 'full', or an integer in [1, k_bins].")
    row_legs = {ps.leg1 for ps in specs}
    col_legs = {ps.leg1 if ps.mode != "leg" else ps.leg2 for ps in specs}
    comps = lambda legs: sum(len(engine.leg_components(l[0], l[1])) for l in legs)
    union_pb = comps(row_legs | col_legs)
    split_pb = comps(row_legs) + (comps(col_legs) if not diagonal else comps(col_legs - row_legs))

    def need(b):
        return union_pb * b if b == k_bins else split_pb * b

    cap = engine.fields_capacity(n, precision, need(bs), free_bytes=free_bytes)
    while bs > 1 and need(bs) > cap:
        bs = (bs + 1) // 2
    if need(bs) > cap:
        raise MemoryError("not enough device memory for one block of shell fields")
    return bs, need(bs)


def bk_sugi_box_multi(meshes, correlation_mode, tracer_type, angu_configs, stat_attrs,
                      precision="f64", block_size=None, shotnoise_ana_all_eff=True):
    """See :func:`bk_sugi_box_submit`; returns the result dicts."""
    return bk_sugi_box_submit(meshes, correlation_mode, tracer_type, angu_configs, stat_attrs, precision,
                              block_size, shotnoise_ana_all_eff)()


def bk_sugi_box_submit(meshes, correlation_mode, tracer_type, angu_configs, stat_attrs,
                       precision="f64", block_size=None, shotnoise_ana_all_eff=True):
    """Sugiyama bispectrum multipoles for several angular configurations of one
    set of painted meshes, sharing the forward transforms, G, the shell fields and
    the FFT shot-noise shells among configurations.

    All device work is enqueued first; the host reads the mode counts and the
    shot-noise shell sums as soon as they are ready (the analytical S3 algebra
    overlaps the remaining GPU work) and the pair sums last.  Returns one
    reference-format result dict per configuration; with a single configuration
    this is ``calculate_bk_sugi_box``.  Returns a function that waits for the
    device results and assembles the dicts, so callers can queue the next
    catalog's work first.
    """
    data_vector_mode = stat_attrs.get("data_vector_mode", "diagonal")
    shotnoise_mode = stat_attrs.get("shotnoise_mode", "ana")
    if data_vector_mode not in ("diagonal", "full"):
        raise ValueError("data_vector_mode must be either 'diagonal' or 'full'.")
    if shotnoise_mode not in ("ana", "fft", "both"):
        raise ValueError("shotnoise_mode must be either 'ana', 'fft', or 'both'.")
    diagonal = data_vector_mode == "diagonal"
    boxsize = np.array(stat_attrs["boxsize"])
    nmesh = np.array(stat_attrs["nmesh"])
    k_min, k_max, k_bins = stat_attrs["k_min"], stat_attrs["k_max"], stat_attrs["k_bins"]
    sampler = stat_attrs["sampler"]
    n = int(nmesh[0])
    L = float(boxsize[0])
    V = boxsize.prod()
    N3 = nmesh.prod()
    vol_per_cell = V / N3
    window = _lib.WINDOW[sampler]
    code, rdt, cdt = engine.PRECISION[precision]
    ctx = _lib.Context.get()

    letters = ["a"] + (["b"] if correlation_mode == "cross" else []) + (["c"] if tracer_type == "abc" else [])
    NZ = {t: stat_attrs["NZ_" + t] for t in letters}
    N_gal = {t: stat_attrs["N_gal_" + t] for t in letters}

    # ---- overdensity spectra: r2c(rho/dV - NZ), compensated (ce:808-837)
    k_edge = np.linspace(k_min, k_max, k_bins + 1)
    # G_00's spectrum: the triple sums see it only at |k| < 2 k_max, so the
    # forward finish of that tracer also writes its band-limited copy
    g_letter = "a" if correlation_mode == "auto" else ("c" if tracer_type == "abc" else "b")
    spec = {}
    for t in letters:
        m = meshes[t]
        k0 = (m.sum_w / float(N3)) / vol_per_cell - NZ[t]
        if t == g_letter:
            spec[t], g_spec = engine.finish_delta_band(m, 1.0 / vol_per_cell, _lib.COMP_SINC, k0, 2.0 * k_max)
        else:
            spec[t] = engine.finish_delta(m, 1.0 / vol_per_cell, _lib.COMP_SINC, k0)
    dev = spec["a"].device

    # ---- mode counts on k and k3 bins (ce:858-865, :1063-1074)
    k_center = 0.5 * (k_edge[1:] + k_edge[:-1])
    k3_edge = np.linspace(2 * k_min, 2 * k_max, k_bins * 2 + 1)[:-1]
    k3_center = 0.5 * (k3_edge[1:] + k3_edge[:-1])
    k3_bins = len(k3_center)
    counts_k = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k_edge)))
    counts_k3 = engine.HostCopy(torch.stack(engine.kbin_counts(n, L, k3_edge)))

    # ---- shot-noise shell sums P(k) Y_L0 on k3 bins (ce:1394-1434) and the
    #      band-limited S3-FFT source field (ce:1187-1210)
    other = spec["a"] if correlation_mode == "auto" else spec.get("b")
    sn_sums = {}
    src_fields = {}
    src_origin = {}
    cfg_info = []
    jobs, sum_keys, src_keys = [], set(), set()
    for (l1, l2, L_) in angu_configs:
        sn0 = N_gal["a"] if (correlation_mode == "auto" and [l1, l2, L_] == [0, 0, 0]) else 0.0
        cfg_info.append(sn0)
        if tracer_type == "abc":
            continue
        key = (L_, sn0)
        need_sum = key not in sum_keys
        need_src = shotnoise_mode in ("fft", "both") and tracer_type != "abb" and sn0 not in src_keys
        if not (need_sum or need_src):
            continue
        if need_sum:
            sum_keys.add(key)
        if need_src:
            src_keys.add(sn0)
        jobs.append((key, L_, sn0, need_sum, need_src))
    # one pass over the modes per two configurations gives their k3-bin sums,
    # source spectra and the sources' x = 0 values
    for j0 in range(0, len(jobs), 2):
        group = jobs[j0:j0 + 2]
        ds = [torch.empty(2 * (k3_bins + 1), dtype=torch.float64, device=dev) for _ in group]
        yls = [angular.harmonic(L_, 0, True) if (L_ != 0 and need_sum) else None
               for (_, L_, _, need_sum, _) in group]
        srcs = [torch.empty(spec["a"].shape, dtype=cdt, device=dev) if need_src else None
                for (*_, need_src) in group]
        any_src = any(x is not None for x in srcs)
        ctx.sn_bins_multi(code, n, L, spec["a"], other, float(V) ** 2, window,
                          [float(sn0) if correlation_mode == "auto" else 0.0 for (_, _, sn0, _, _) in group],
                          yls, k3_edge, ds, srcs, band=2.0 * k_max if any_src else 0.0)
        for (key, _, sn0, need_sum, need_src), d, src_spec in zip(group, ds, srcs):
            if need_sum:
                sn_sums[key] = engine.HostCopy(d)
            if need_src:
                fld = torch.empty(n * n * n, dtype=rdt, device=dev)
                ctx.c2r(code, n, 1, src_spec, fld)
                if precision == "f32":
                    # x = 0 cell added in FP64 (engine.origin_correction)
                    src_origin[sn0] = engine.HostCopy(d[2 * k3_bins:])
                    fld.narrow(0, 0, 1).zero_()
                src_fields[sn0] = fld
        del srcs

    # ---- signal: G_00 = Re c2r(delta) band-limited to |k| < 2 k_max (the only
    #      modes the triple sums see), shell fields, pair sums (ce:867-1061)
    G = torch.empty(n * n * n, dtype=rdt, device=dev)
    ctx.c2r(code, n, 1, g_spec, G)
    del g_spec
    specs, per_cfg = [], []
    for (l1, l2, L_) in angu_configs:
        cfgs, tj = angular.magnetic_configs_box(l1, l2, L_)
        entries = []
        for ss, (m1, m2, _) in enumerate(cfgs):
            entries.append((len(specs), (m1, m2), tj[ss]))
            specs.append(_legs_for_signal(l1, l2, m1, m2, correlation_mode, tracer_type))
        per_cfg.append(entries)
    free_bytes = engine.free_device_bytes()
    bs, capacity = _plan_blocks(specs, k_bins, n, precision, block_size, diagonal, free_bytes)
    sf = engine.ShellFields(n, L, k_edge, precision, spec["a"], spec.get("b"), capacity=capacity)
    signal = engine.pair_sums([(G, specs)], sf, k_bins, diagonal, bs)[0]
    del sf, G

    # ---- S3 by FFT: data-independent shells conj(Y) mask on a unit spectrum,
    #      shared by every configuration, contracted with each configuration's
    #      source field (ce:1182-1384)
    s3_groups, s3_index = [], {}
    for ci, (l1, l2, L_) in enumerate(angu_configs):
        sn0 = cfg_info[ci]
        if sn0 not in src_fields:
            continue
        cfgs, tj = angular.magnetic_configs_box(l1, l2, L_)
        s3_index[ci] = len(s3_groups)
        s3_groups.append((src_fields[sn0], [_legs_for_s3fft(l1, l2, m1, m2) for (m1, m2, _) in cfgs]))
    s3fft = {}
    shell_origin = None
    if s3_groups:
        all_sp = [ps for (_, sp) in s3_groups for ps in sp]
        bsf, capf = _plan_blocks(all_sp, k_bins, n, precision, block_size, diagonal, free_bytes)
        if engine.UNIT_SHELL_CACHE and bsf >= k_bins:
            sfu = engine.unit_shells(n, L, k_edge, precision, capf)
        else:
            sfu = engine.ShellFields(n, L, k_edge, precision, None, None, capacity=capf)
        outs = engine.pair_sums(s3_groups, sfu, k_bins, diagonal, bsf)
        s3fft = {ci: outs[gi] for ci, gi in s3_index.items()}
        del sfu
        if src_origin:
            legs = [ps.leg1 for ps in all_sp] + [ps.leg2 for ps in all_sp if ps.mode == "leg"]
            shell_origin = engine.unit_shell_origin(n, L, k_edge, precision, legs)

    def finalize(n_gal=None, sn_unit=None):
        """Host algebra once the device work is queued.  ``n_gal`` (auto
        correlation): the catalog's real count when the device work ran with
        another one (a padded CUDA-graph capture, zero-weight padding); the
        analytic shot-noise sums are then moved from the captured sn0 to n_gal
        with ``sn_unit[L]``, the k3-bin sums of the same kernel for a zero
        spectrum and sn0 = 1 (the sums are linear in sn0)."""
        return _bk_box_results(
            angu_configs, tracer_type, correlation_mode, diagonal, shotnoise_mode, shotnoise_ana_all_eff, k_bins,
            k_edge, k3_center, nmesh, V, vol_per_cell, N_gal, counts_k, counts_k3, sn_sums, cfg_info, s3fft,
            s3_groups, s3_index, src_origin, shell_origin, signal, per_cfg, n_gal, sn_unit)

    return finalize


def _bk_box_results(angu_configs, tracer_type, correlation_mode, diagonal, shotnoise_mode, shotnoise_ana_all_eff,
                    k_bins, k_edge, k3_center, nmesh, V, vol_per_cell, N_gal, counts_k, counts_k3, sn_sums,
                    cfg_info, s3fft, s3_groups, s3_index, src_origin, shell_origin, signal, per_cfg,
                    n_gal=None, sn_unit=None):
    """Host algebra of bk_sugi_box_multi, run once the device work is queued."""
    sn_captured = list(cfg_info)
    if n_gal is not None and n_gal != N_gal["a"]:
        if correlation_mode != "auto":
            raise ValueError("a count override is defined for auto correlations only")
        if shotnoise_mode != "ana" and any(sn_captured):
            raise ValueError("a count override needs shotnoise_mode 'ana' (the FFT S3 source depends on the count)")
        N_gal = {"a": int(n_gal)}
        cfg_info = [float(n_gal) if sn0 else 0.0 for sn0 in sn_captured]
    k_center = 0.5 * (k_edge[1:] + k_edge[:-1])
    k3_bins = len(k3_center)
    ck = counts_k.get()
    k_num, k_eff = ck[0].copy(), ck[1] / ck[0]
    c3 = counts_k3.get()
    k_num_k3, k3_eff = c3[0].copy(), c3[1] / c3[0]

    results = []
    sig = None
    for ci, (l1, l2, L_) in enumerate(angu_configs):
        N_ells = (2 * l1 + 1) * (2 * l2 + 1) * (2 * L_ + 1)
        H_ells = angular.wigner3j(l1, l2, L_, 0, 0, 0)
        cfgs, tj = angular.magnetic_configs_box(l1, l2, L_)
        SN3_fft = None
        if tracer_type == "abc":
            SN0, SN1, SN2, SN3 = 0.0, 0.0, 0.0, 0.0
        else:
            SN0 = cfg_info[ci]
            dd = sn_sums[(L_, sn_captured[ci])].get()[:2 * k3_bins]
            if SN0 != sn_captured[ci]:
                dd = dd + (SN0 - sn_captured[ci]) * np.asarray(sn_unit[L_])[:2 * k3_bins]
            total_sum = dd[0::2] + 1j * dd[1::2]
            SN1, SN2 = 0.0, 0.0
            if l1 == L_ and l2 == 0:
                if correlation_mode == "auto":
                    SN1 = (total_sum / k_num_k3)[: len(k_center)]
                    SN1 *= 2 * L_ + 1
                    if l1 == 0:
                        SN2 = SN1.copy()
                elif correlation_mode == "cross" and tracer_type == "abb":
                    SN1 = (total_sum / k_num_k3)[: len(k_center)]
                    SN1 *= 2 * L_ + 1
            if not diagonal:
                SN1_full = np.zeros((k_bins, k_bins)).astype("c16")
                SN2_full = np.zeros((k_bins, k_bins)).astype("c16")
                if np.isscalar(SN1) or np.ndim(SN1) == 0:
                    SN1_full[:] = SN1
                else:
                    for i in range(k_bins):
                        SN1_full[i, :] = SN1[i]
                if np.isscalar(SN2) or np.ndim(SN2) == 0:
                    SN2_full[:] = SN2
                else:
                    for i in range(k_bins):
                        SN2_full[:, i] = SN2[i]
                SN1, SN2 = SN1_full, SN2_full

            def s3_ana():
                if tracer_type == "abb":
                    return 0.0
                if shotnoise_ana_all_eff:
                    q = angular.q_ells_matrix(k_eff, l1, l2, L_, k3_eff)
                else:
                    q = angular.q_ells_matrix(k_center, l1, l2, L_, k3_center)
                return angular.s3_analytic(total_sum, k_num_k3, k_edge, k3_center, q, diagonal) * (H_ells * N_ells)

            def s3_fft():
                if tracer_type == "abb":
                    return np.zeros((k_bins, k_bins) if not diagonal else k_bins, dtype="complex128")
                ss_list = s3fft[ci].result()
                s3 = np.zeros((k_bins, k_bins) if not diagonal else k_bins, dtype="complex128")
                specs_ci = s3_groups[s3_index[ci]][1]
                for ss, (m1, m2, _) in enumerate(cfgs):
                    S = ss_list[ss]
                    if src_origin:
                        v0 = src_origin[cfg_info[ci]].get()
                        S = S + engine.origin_correction(specs_ci[ss], shell_origin, complex(v0[0], 0.0),
                                                         k_bins, diagonal)
                    if diagonal:
                        sub = np.zeros(k_bins, dtype="complex128")
                        ok = k_num > 0
                        sub[ok] = tj[ss] * S[ok] / (k_num[ok] ** 2)
                    else:
                        sub = np.zeros((k_bins, k_bins), dtype="complex128")
                        ok = np.outer(k_num > 0, k_num > 0)
                        with np.errstate(divide="ignore", invalid="ignore"):
                            sub[ok] = (tj[ss] * S / np.outer(k_num, k_num))[ok]
                    s3 += sub if (m1, m2) == (0, 0) else 2.0 * np.real(sub)
                s3 *= H_ells * N_ells
                s3 *= 1 / nmesh.prod()
                return s3

            if shotnoise_mode == "ana":
                SN3 = s3_ana()
            elif shotnoise_mode == "fft":
                SN3 = s3_fft()
            else:
                SN3 = s3_ana()
                SN3_fft = s3_fft()

        if sig is None:
            sig = signal.result()
        total_res = np.zeros(k_bins if diagonal else (k_bins, k_bins)).astype("complex128")
        for (idx, (m1, m2), three_j) in per_cfg[ci]:
            sub = three_j * sig[idx]
            total_res += sub if (m1, m2) == (0, 0) else 2 * np.real(sub)

        # normalisation (ce:1495-1548)
        if correlation_mode == "auto":
            I_norm = (N_gal["a"] ** 3) / (V ** 2)
        elif tracer_type == "aab":
            I_norm = (N_gal["a"] ** 2 * N_gal["b"]) / (V ** 2)
        elif tracer_type == "abb":
            I_norm = (N_gal["a"] * N_gal["b"] ** 2) / (V ** 2)
        else:
            I_norm = (N_gal["a"] * N_gal["b"] * N_gal["c"]) / (V ** 2)
        total_shot_noise = SN0 + SN1 + SN2 + SN3
        total_res *= N_ells * H_ells / I_norm
        if not diagonal:
            total_res *= V ** 2 / np.outer(k_num[:k_bins], k_num[:k_bins])
        else:
            total_res *= V ** 2 / (k_num[: len(total_res)]) ** 2
        total_res *= vol_per_cell
        total_shot_noise *= 1 / I_norm
        final_bk = total_res - total_shot_noise
        sn_terms = {"SN0": SN0 / I_norm, "SN1": SN1 / I_norm, "SN2": SN2 / I_norm, "SN3": SN3 / I_norm}
        if shotnoise_mode == "both":
            # the reference divides None by I_norm here for tracer "abc" (TypeError)
            sn_terms["SN3_FFT"] = SN3_fft / I_norm
        results.append({
            "B_sugi": final_bk, "SN_terms": sn_terms, "I_norm": I_norm, "Shot_noise": total_shot_noise,
            "Bk_raw": total_res, "k_eff": k_eff, "nmodes": k_num,
        })
    return results


def _q_ells_center(i, j, k_center, k_min, k_max, k_bins, l1, l2, L):
    """q_l with bin-centre wavenumbers (math_evaluator.py:560-589)."""
    k3_edge = np.linspace(2 * k_min, 2 * k_max, k_bins * 2 + 1)[:-1]
    k3_center = 0.5 * (k3_edge[1:] + k3_edge[:-1])
    q = np.zeros(len(k3_center))
    lmin = min(l1, l2)
    k1, k2 = k_center[i], k_center[j]
    for nn in range(-lmin, lmin + 1):
        tj = angular.wigner3j(l1, l2, L, nn, -nn, 0)
        a13 = np.zeros(len(k3_center))
        a23 = np.zeros(len(k3_center))
        for t, k3 in enumerate(k3_center):
            if abs(k1 - k2) <= k3 <= (k1 + k2):
                a13[t] = angular.assoc_legendre(l1, nn, (k3 ** 2 + k1 ** 2 - k2 ** 2) / (2 * k1 * k3))
                a23[t] = angular.assoc_legendre(l2, -nn, (k3 ** 2 + k2 ** 2 - k1 ** 2) / (2 * k2 * k3))
        a13 *= (-1) ** (l1 + nn)
        a23 *= (-1) ** (l2 - nn)
        q += (-1) ** nn * tj * a13 * a23
    return q


def calculate_bk_sugi_box(rfield_a, rfield_b, rfield_c, correlation_mode, stat_attrs, comm=None, **kwargs):
    """Sugiyama bispectrum multipole in a periodic box (clustering_estimator.py:749-1555)."""
    precision = _precision(stat_attrs, kwargs)
    tracer_type = stat_attrs["tracer_type"]
    meshes = {"a": rfield_a}
    if correlation_mode == "cross":
        meshes["b"] = rfield_b
        if tracer_type == "abc":
            meshes["c"] = rfield_c
    block_size = stat_attrs.get("block_size", 1 if stat_attrs.get("data_vector_mode", "diagonal") == "diagonal" else "full")
    res = bk_sugi_box_multi(meshes, correlation_mode, tracer_type, [tuple(stat_attrs["angu_config"])], stat_attrs,
                            precision=precision, block_size=block_size,
                            shotnoise_ana_all_eff=kwargs.get("shotnoise_ana_all_eff", True))
    logging.getLogger(__name__).info("bk_sugi box finished")
    return res[0]
