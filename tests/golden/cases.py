"""Small box workloads pinned by golden vectors from the reference.

Each case is a reference config dict (keys as in the reference's config files)
plus the seeds of its synthetic catalogs.  Catalogs are regenerated from the
seeds (numpy PCG64 is deterministic) and checked against the stored position
checksum, so the fixtures only hold results.
"""
from __future__ import annotations

import copy
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_BASE = dict(
    geometry="box-like",
    rsd=[0, 0, 1],
    apply_rsd=False,
    cosmology={"h": 0.6766, "Omega0": 0.31},
    redshift_box=0.0,
    compensation=True,
)

# (name, config overrides, catalogs: {letter: (seed, n_particles, weighted)})
CASES = [
    ("pk_auto_cic_il", dict(statistic="pk", correlation_mode="auto", nmesh=[32] * 3,
                            boxsize=[1000.0] * 3, sampler="cic", interlaced=True,
                            k_min=0.005, k_max=0.095, k_bins=9, poles=[0, 2, 4]),
     {"a": (11, 20000, False)}),
    ("pk_cross_tsc_noil", dict(statistic="pk", correlation_mode="cross", nmesh=[32] * 3,
                               boxsize=[800.0] * 3, sampler="tsc", interlaced=False,
                               k_min=0.01, k_max=0.11, k_bins=5, poles=[0, 1, 2], rsd=[0, 1, 0]),
     {"a": (12, 15000, True), "b": (13, 12000, False)}),
    ("pk_auto_ngp_k0", dict(statistic="pk", correlation_mode="auto", nmesh=[32] * 3,
                            boxsize=[1000.0] * 3, sampler="ngp", interlaced=True,
                            k_min=0.0, k_max=0.09, k_bins=6, poles=[0, 2]),
     {"a": (14, 20000, False)}),
    ("pk_auto_pcs_noil", dict(statistic="pk", correlation_mode="auto", nmesh=[32] * 3,
                              boxsize=[1000.0] * 3, sampler="pcs", interlaced=False,
                              k_min=0.005, k_max=0.095, k_bins=9, poles=[0, 2, 4],
                              rsd=[0.6, 0.0, 0.8]),
     {"a": (15, 20000, False)}),
    ("bk_diag_000_tsc", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="tsc", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[0, 0, 0],
                             data_vector_mode="diagonal", shotnoise_mode="ana"),
     {"a": (21, 20000, False)}),
    ("bk_diag_202_tsc", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="tsc", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[2, 0, 2],
                             data_vector_mode="diagonal", shotnoise_mode="both"),
     {"a": (21, 20000, False)}),
    ("bk_diag_110_cic", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="cic", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[1, 1, 0],
                             data_vector_mode="diagonal", shotnoise_mode="fft"),
     {"a": (22, 20000, True)}),
    ("bk_full_000_pcs", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="pcs", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[0, 0, 0],
                             data_vector_mode="full", shotnoise_mode="both", block_size=2),
     {"a": (23, 20000, False)}),
    ("bk_full_202_pcs", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="pcs", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[2, 0, 2],
                             data_vector_mode="full", shotnoise_mode="both", block_size="full"),
     {"a": (23, 20000, False)}),
    ("bk_full_112_cic", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="cic", interlaced=False,
                             k_min=0.005, k_max=0.045, k_bins=3, angu_config=[1, 1, 2],
                             data_vector_mode="full", shotnoise_mode="both", block_size=1),
     {"a": (24, 20000, False)}),
    ("bk_full_220_ngp", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="ngp", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=3, angu_config=[2, 2, 0],
                             data_vector_mode="full", shotnoise_mode="fft"),
     {"a": (25, 20000, False)}),
    ("bk_cross_aab_full", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="aab",
                               nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="tsc", interlaced=True,
                               k_min=0.005, k_max=0.045, k_bins=3, angu_config=[0, 0, 0],
                               data_vector_mode="full", shotnoise_mode="both"),
     {"a": (26, 15000, False), "b": (27, 12000, True)}),
    ("bk_cross_abb_diag", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="abb",
                               nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="cic", interlaced=True,
                               k_min=0.005, k_max=0.045, k_bins=4, angu_config=[2, 0, 2],
                               data_vector_mode="diagonal", shotnoise_mode="both"),
     {"a": (26, 15000, False), "b": (27, 12000, True)}),
    ("bk_cross_abc_full", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="abc",
                               nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="tsc", interlaced=False,
                               k_min=0.005, k_max=0.045, k_bins=3, angu_config=[2, 0, 2],
                               data_vector_mode="full", shotnoise_mode="ana"),
     {"a": (26, 15000, False), "b": (27, 12000, True), "c": (28, 10000, False)}),
    # box catalogs in FITS files with velocity columns: the reference applies its
    # redshift-space shift (catalog_processor.py:410-433, :648-693); "_format"
    # names the file layout (lower- or upper-case column names, weights)
    ("bk_fits_rsd_tsc", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                             nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="tsc", interlaced=True,
                             k_min=0.005, k_max=0.045, k_bins=4, angu_config=[2, 0, 2],
                             data_vector_mode="diagonal", shotnoise_mode="both", apply_rsd=True,
                             redshift_box=0.5, rsd=[0, 0, 1], _format="fits_lower"),
     {"a": (29, 20000, False)}),
    ("pk_fits_rsd_upper_w", dict(statistic="pk", correlation_mode="auto", nmesh=[32] * 3,
                                 boxsize=[800.0] * 3, sampler="pcs", interlaced=True, k_min=0.005,
                                 k_max=0.115, k_bins=8, poles=[0, 2, 4], apply_rsd=True, redshift_box=1.0,
                                 rsd=[0, 1, 0], cosmology={"h": 0.7, "Omega0": 0.3}, _format="fits_upper"),
     {"a": (30, 20000, True)}),
    ("pk_fits_norsd_cross", dict(statistic="pk", correlation_mode="cross", nmesh=[32] * 3,
                                 boxsize=[1000.0] * 3, sampler="cic", interlaced=False, k_min=0.005,
                                 k_max=0.095, k_bins=9, poles=[0, 2], apply_rsd=False, _format="fits_lower"),
     {"a": (31, 15000, True), "b": (32, 12000, False)}),
    # box catalogs in HDF5 files (h5_reader, catalog_processor.py:16-88): float64,
    # big-endian, float32 and chunked/deflated columns
    ("bk_h5_rsd_full", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                            nmesh=[32] * 3, boxsize=[1000.0] * 3, sampler="cic", interlaced=True,
                            k_min=0.005, k_max=0.045, k_bins=3, angu_config=[0, 0, 0],
                            data_vector_mode="full", shotnoise_mode="ana", apply_rsd=True,
                            redshift_box=0.3, rsd=[1, 0, 0], _format="h5_lower"),
     {"a": (33, 20000, True)}),
    ("pk_h5_upper_norsd", dict(statistic="pk", correlation_mode="auto", nmesh=[32] * 3,
                               boxsize=[1000.0] * 3, sampler="tsc", interlaced=True, k_min=0.005,
                               k_max=0.095, k_bins=9, poles=[0, 2, 4], apply_rsd=False, _format="h5_upper"),
     {"a": (34, 20000, False)}),
]


# Survey-like cases (FITS catalogs, RA/DEC/Z columns).  Catalog spec per tracer:
# (seed, n_data, n_randoms, boss_weights); the survey occupies RA 150-180 deg,
# DEC 10-35 deg, 0.4 < z < 0.6, inside a 1000 Mpc/h box.
_SURVEY_BASE = dict(
    geometry="survey-like",
    column_names=["RA", "DEC", "Z", "WEIGHT_FKP", "WEIGHT_SYSTOT", "WEIGHT_NOZ", "WEIGHT_CP", "NZ"],
    cosmology={"h": 0.6766, "Omega0": 0.31},
    compensation=True,
    nmesh=[32] * 3,
    boxsize=[1000.0] * 3,
    z_range=[0.42, 0.58],
    comp_weight_plan={"scheme": "boss", "name_alias": None},
    alpha_scheme="pypower",
)
_SA = {"a": (41, 20000, 100000, True)}
_SAB = {"a": (41, 20000, 100000, True), "b": (42, 15000, 80000, True)}
_SABC = {"a": (41, 20000, 100000, True), "b": (42, 15000, 80000, True), "c": (43, 12000, 70000, True)}

SURVEY_CASES = [
    ("sv_pk_auto_tsc_particle", dict(statistic="pk", correlation_mode="auto", sampler="tsc",
                                     interlaced=True, k_min=0.0, k_max=0.09, k_bins=9, poles=[0, 2, 4],
                                     normalization_scheme="particle"), _SA),
    ("sv_pk_cross_cic_mixed", dict(statistic="pk", correlation_mode="cross", sampler="cic",
                                   interlaced=False, k_min=0.005, k_max=0.085, k_bins=8, poles=[0, 1, 2],
                                   normalization_scheme="mixed-mesh", alpha_scheme="nbodykit",
                                   z_range=None, comp_weight_plan={"scheme": None, "name_alias": None}),
     _SAB),
    ("sv_pk_auto_pcs_compare", dict(statistic="pk", correlation_mode="auto", sampler="pcs",
                                    interlaced=True, k_min=0.0, k_max=0.09, k_bins=6, poles=[0, 2, 4, 6, 8],
                                    normalization_scheme="mixed-mesh", high_order_mode="compare",
                                    comp_weight_plan={"scheme": "eboss", "name_alias": None}), _SA),
    ("sv_pk_auto_ngp_fast", dict(statistic="pk", correlation_mode="auto", sampler="ngp",
                                 interlaced=True, k_min=0.0, k_max=0.09, k_bins=6, poles=[0, 2, 4],
                                 normalization_scheme="particle", high_order_mode="fast"), _SA),
    ("sv_bk_000_diag_tsc", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                                sampler="tsc", interlaced=True, k_min=0.005, k_max=0.045, k_bins=4,
                                angu_config=[0, 0, 0], data_vector_mode="diagonal", shotnoise_mode="both",
                                normalization_scheme="particle"), _SA),
    ("sv_bk_202_full_pcs_mixed", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                                      sampler="pcs", interlaced=True, k_min=0.005, k_max=0.045, k_bins=4,
                                      angu_config=[2, 0, 2], data_vector_mode="full", shotnoise_mode="both",
                                      block_size=2, normalization_scheme="mixed-mesh"), _SA),
    ("sv_bk_110_diag_cic_mesh", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                                     sampler="cic", interlaced=False, k_min=0.005, k_max=0.045, k_bins=4,
                                     angu_config=[1, 1, 0], data_vector_mode="diagonal",
                                     shotnoise_mode="fft", normalization_scheme="mesh"), _SA),
    ("sv_bk_112_full_ngp", dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                                sampler="ngp", interlaced=True, k_min=0.005, k_max=0.045, k_bins=3,
                                angu_config=[1, 1, 2], data_vector_mode="full", shotnoise_mode="both",
                                normalization_scheme="particle", alpha_scheme="nbodykit"), _SA),
    ("sv_bk_aab_000_full", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="aab",
                                sampler="tsc", interlaced=True, k_min=0.005, k_max=0.045, k_bins=3,
                                angu_config=[0, 0, 0], data_vector_mode="full", shotnoise_mode="both",
                                normalization_scheme="mixed-mesh"), _SAB),
    ("sv_bk_abb_202_diag", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="abb",
                                sampler="cic", interlaced=True, k_min=0.005, k_max=0.045, k_bins=4,
                                angu_config=[2, 0, 2], data_vector_mode="diagonal", shotnoise_mode="ana",
                                normalization_scheme="mixed-mesh"), _SAB),
    # cosmology without Omega0: the reference converts redshifts with Planck18
    # (catalog_processor.py:610-625) and still multiplies by the config's h
    ("sv_pk_auto_planck18", dict(statistic="pk", correlation_mode="auto", sampler="cic", interlaced=True,
                                 k_min=0.005, k_max=0.085, k_bins=8, poles=[0, 2], cosmology={"h": 0.6766},
                                 normalization_scheme="particle"), _SA),
    ("sv_bk_abc_000_diag", dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="abc",
                                sampler="tsc", interlaced=False, k_min=0.005, k_max=0.045, k_bins=4,
                                angu_config=[0, 0, 0], data_vector_mode="diagonal", shotnoise_mode="ana",
                                normalization_scheme="mixed-mesh"), _SABC),
]


def build_survey_case(name, workdir):
    """Write the survey case's FITS catalogs under ``workdir``; return (config, checksums)."""
    from cosmonpc_b200 import mocks

    for cname, over, cats in SURVEY_CASES:
        if cname != name:
            continue
        cfg = copy.deepcopy(_SURVEY_BASE)
        cfg.update(copy.deepcopy(over))
        catalogs = {"data_a": None, "randoms_a": None, "data_b": None, "randoms_b": None}
        sums = {}
        os.makedirs(workdir, exist_ok=True)
        for letter, (seed, nd, nr, boss) in cats.items():
            d, r = mocks.survey_catalogs(nd, nr, seed, boss_weights=boss)
            for kind, cols in (("data", d), ("randoms", r)):
                path = os.path.join(workdir, "%s_%s_%s.fits" % (name, kind, letter))
                mocks.write_fits_catalog(path, cols)
                catalogs["%s_%s" % (kind, letter)] = path
                sums["%s_%s" % (kind, letter)] = float(sum(np.sum(v) for v in cols.values()))
        cfg["catalogs"] = catalogs
        cfg["output_dir"] = os.path.join(workdir, "out_" + name)
        return cfg, sums
    raise KeyError(name)


def catalog_positions(seed, n_particles, boxsize):
    from cosmonpc_b200.mocks import lognormal_box

    return lognormal_box(n_particles, boxsize, seed, grid=32)


def catalog_velocities(seed, n):
    """Peculiar velocities in km/s, N(0, 300) per axis."""
    rng = np.random.Generator(np.random.PCG64(seed + 2000))
    return rng.normal(0.0, 300.0, (n, 3))


def catalog_weights(seed, n):
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    return 0.5 + rng.random(n)


def build_case(name, workdir):
    """Write the case's catalogs under ``workdir`` and return (config, checksums)."""
    if name.startswith("sv_"):
        return build_survey_case(name, workdir)
    for cname, over, cats in CASES:
        if cname != name:
            continue
        cfg = copy.deepcopy(_BASE)
        cfg.update(copy.deepcopy(over))
        fmt = cfg.pop("_format", "npy")
        L = cfg["boxsize"][0]
        weighted = any(v[2] for v in cats.values())
        cfg["column_names"] = ["x", "y", "z", "w"] if weighted else ["x", "y", "z"]
        if fmt.startswith(("fits", "h5")):
            names = ["x", "y", "z", "vx", "vy", "vz"]
            if fmt.endswith("_upper"):
                names = [c.upper() for c in names]
            # an extra column the reference must ignore, and the weight column
            cfg["column_names"] = names + (["w"] if weighted else []) + ["ID"]
        catalogs = {"data_a": None, "randoms_a": None, "data_b": None, "randoms_b": None}
        sums = {}
        os.makedirs(workdir, exist_ok=True)
        for letter, (seed, npart, wflag) in cats.items():
            pos = catalog_positions(seed, npart, L)
            arr = pos
            if weighted:
                w = catalog_weights(seed, len(pos)) if wflag else np.ones(len(pos))
                arr = np.column_stack([pos, w])
            if fmt.startswith("fits"):
                from cosmonpc_b200 import fits

                vel = catalog_velocities(seed, len(pos))
                cols = {nm: v for nm, v in zip(cfg["column_names"][:6], [pos[:, 0], pos[:, 1], pos[:, 2],
                                                                           vel[:, 0], vel[:, 1], vel[:, 2]])}
                if weighted:
                    cols["w"] = arr[:, 3]
                cols["ID"] = np.arange(len(pos), dtype=np.int64)
                cols["MASS"] = np.full(len(pos), 1e12, dtype=np.float32)  # not requested
                path = os.path.join(workdir, "%s_%s.fits" % (name, letter))
                fits.write_table(path, cols)
                arr = np.column_stack([arr, vel])
            elif fmt.startswith("h5"):
                from cosmonpc_b200 import hdf5

                vel = catalog_velocities(seed, len(pos))
                n6 = cfg["column_names"][:6]
                cols = {n6[0]: pos[:, 0], n6[1]: pos[:, 1].astype(">f8"), n6[2]: pos[:, 2],
                        n6[3]: vel[:, 0].astype(np.float32), n6[4]: vel[:, 1], n6[5]: vel[:, 2]}
                if weighted:
                    cols["w"] = arr[:, 3]
                cols["ID"] = np.arange(len(pos), dtype=np.int64)
                path = os.path.join(workdir, "%s_%s.h5" % (name, letter))
                hdf5.write_columns(path, cols, chunked={n6[2]: 4096, n6[5]: 3000})
                v32 = vel.copy()
                v32[:, 0] = v32[:, 0].astype(np.float32)
                arr = np.column_stack([arr, v32])
            else:
                path = os.path.join(workdir, "%s_%s.npy" % (name, letter))
                np.save(path, arr)
            catalogs["data_" + letter] = path
            sums[letter] = float(np.sum(arr))
        cfg["catalogs"] = catalogs
        cfg["output_dir"] = os.path.join(workdir, "out_" + name)
        return cfg, sums
    raise KeyError(name)


# survey-only result / attribute keys kept in the fixtures
SURVEY_KEYS = ("P4b", "P6b", "P8b", "N0", "I_rand", "I_data", "I_mesh", "boxcenter")


def flatten_result(res):
    """Numeric keys of a result dict as a flat {name: ndarray} mapping."""
    out = {}
    for k, v in res.items():
        if k == "SN_terms":
            for kk, vv in v.items():
                out["SN_terms." + kk] = np.asarray(vv)
        elif k in ("B_sugi", "Bk_raw", "Shot_noise", "I_norm", "k_eff", "nmodes", "k_num",
                   "P_shot") or (k.startswith("P") and k[1:].isdigit()):
            out[k] = np.asarray(v)
        elif (k in SURVEY_KEYS or k.startswith(("alpha_", "I_33_", "S_LM_"))) and not isinstance(v, str):
            out[k] = np.asarray(v)
    return out
