"""The benchmark workloads at their own sizes, pinned by golden vectors of the
reference itself.

Each entry is a reference config dict for one ``run_stats`` call plus the recipe
of its seeded synthetic catalogs.  ``make_golden_configs.py`` runs the
unmodified reference on them (single-rank stand-ins, ``ref_shims.py``) and
stores the numeric result keys as ``cfg_<name>.npz``; the GPU tests run the
CUDA path on the same catalogs (regenerated from the seeds and checked against
the stored checksums) and compare.

Workloads (seeds: base seed 20261203 + the workload number; mocks: + 5 + i):

1. pk box auto, 64^3, 1000 Mpc/h, 1e5 lognormal particles, CIC interlaced,
   poles [0, 2, 4], 19 bins 0.005-0.195 h/Mpc (k_max kept below the Nyquist
   frequency 0.2011, which the reference enforces, task_executor.py:35-40).
2. bk_sugi box auto diagonal, 128^3, 1000 Mpc/h, 1e6 particles, TSC interlaced,
   (0,0,0), (2,0,2) and (1,1,0), 19 bins 0.01-0.20, shot noise "ana".
3. bk_sugi box auto full, 256^3, 2000 Mpc/h, 4e6 particles, PCS interlaced,
   (0,0,0) and (2,0,2), the full 20 x 20 data vector over 0.01-0.20
   (2 k_max < k_Nyquist, task_executor.py:192-196), shot noise "both".
4. survey cross at a tenth of the catalog sizes and 256^3 instead of 512^3:
   2e5 data points and 4e6 randoms with RA in [100, 260] deg, sin(DEC) uniform
   over [0, 60] deg, Z ~ N(0.5, 0.1) clipped to [0.2, 0.8], tracer b an
   independent clustered catalog of half the data count sharing the randoms,
   box 3500 Mpc/h (the footprint wraps, as in the full workload), TSC
   interlaced, mixed-mesh normalisation; pk cross [0, 2, 4] (20 bins
   0.005-0.205) and bk_sugi aab (0,0,0) and (2,0,2) diagonal (10 bins
   0.01-0.11).
5. one mock of each shape class of the batched-mocks workload: a Poisson
   count of mean 1.5e6 at 128^3/1000, 192^3/1500 and 256^3/2000 Mpc/h, CIC
   interlaced, pk [0, 2, 4] and bk_sugi (0,0,0) diagonal over 15 bins
   0.01-0.16.
"""
from __future__ import annotations

import copy
import os

import numpy as np

BASE_SEED = 20261203

_BOX = dict(geometry="box-like", rsd=[0, 0, 1], apply_rsd=False, cosmology={"h": 0.6766, "Omega0": 0.31},
            redshift_box=0.0, compensation=True, column_names=["x", "y", "z"])

# name -> (config overrides, box catalog (n_particles, boxsize, seed) or survey recipe)
CONFIG_CASES = {}


def _add_box(name, over, npart, L, seed):
    n = over.pop("n")
    CONFIG_CASES[name] = (dict(_BOX, **over, nmesh=[n] * 3, boxsize=[L] * 3), ("box", npart, L, seed))


_add_box("c1_pk_64", dict(n=64, statistic="pk", correlation_mode="auto", sampler="cic", interlaced=True,
                          k_min=0.005, k_max=0.195, k_bins=19, poles=[0, 2, 4]), 100_000, 1000.0, BASE_SEED + 1)
for _cfg in ([0, 0, 0], [2, 0, 2], [1, 1, 0]):
    _add_box("c2_bk_diag_128_%d%d%d" % tuple(_cfg),
             dict(n=128, statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa", sampler="tsc",
                  interlaced=True, k_min=0.01, k_max=0.20, k_bins=19, angu_config=list(_cfg),
                  data_vector_mode="diagonal", shotnoise_mode="ana"), 1_000_000, 1000.0, BASE_SEED + 2)
for _cfg in ([0, 0, 0], [2, 0, 2]):
    _add_box("c3_bk_full_256_%d%d%d" % tuple(_cfg),
             dict(n=256, statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa", sampler="pcs",
                  interlaced=True, k_min=0.01, k_max=0.20, k_bins=20, angu_config=list(_cfg),
                  data_vector_mode="full", shotnoise_mode="both"), 4_000_000, 2000.0, BASE_SEED + 3)
for _i, (_n, _L) in enumerate(((128, 1000.0), (192, 1500.0), (256, 2000.0))):
    _seed = BASE_SEED + 5 + 32 * _i
    _add_box("c5_mock_%d_pk" % _n, dict(n=_n, statistic="pk", correlation_mode="auto", sampler="cic",
                                        interlaced=True, k_min=0.01, k_max=0.16, k_bins=15, poles=[0, 2, 4]),
             1_500_000, _L, _seed)
    _add_box("c5_mock_%d_bk000" % _n, dict(n=_n, statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa",
                                           sampler="cic", interlaced=True, k_min=0.01, k_max=0.16, k_bins=15,
                                           angu_config=[0, 0, 0], data_vector_mode="diagonal",
                                           shotnoise_mode="ana"), 1_500_000, _L, _seed)

SURVEY4 = dict(scale=0.1, n_data=2_000_000, n_randoms=40_000_000, seed=BASE_SEED + 4,
               geo=dict(ra=(100.0, 260.0), dec=(0.0, 60.0), z_mu=0.5, z_sigma=0.1, z_clip=(0.2, 0.8)))
_SV = dict(geometry="survey-like", column_names=["RA", "DEC", "Z", "WEIGHT_FKP", "NZ"],
           cosmology={"h": 0.676, "Omega0": 0.31}, compensation=True, nmesh=[256] * 3, boxsize=[3500.0] * 3,
           z_range=[0.2, 0.8], sampler="tsc", interlaced=True, comp_weight_plan={"scheme": None, "name_alias": None},
           alpha_scheme="pypower", normalization_scheme="mixed-mesh")
CONFIG_CASES["c4_sv_pk_cross"] = (dict(_SV, statistic="pk", correlation_mode="cross", k_min=0.005, k_max=0.205,
                                       k_bins=20, poles=[0, 2, 4]), ("survey",))
for _cfg in ([0, 0, 0], [2, 0, 2]):
    CONFIG_CASES["c4_sv_bk_aab_%d%d%d" % tuple(_cfg)] = (
        dict(_SV, statistic="bk_sugi", correlation_mode="cross", tracer_type="aab", k_min=0.01, k_max=0.11,
             k_bins=10, angu_config=list(_cfg), data_vector_mode="diagonal", shotnoise_mode="ana"), ("survey",))


def survey4_catalogs(workdir):
    """Write the scaled survey workload's FITS catalogs; returns (catalogs dict, checksums)."""
    from cosmonpc_b200 import mocks

    s = SURVEY4
    nd, nr = int(s["n_data"] * s["scale"]), int(s["n_randoms"] * s["scale"])
    d_a, r_a = mocks.survey_catalogs(nd, nr, s["seed"], **s["geo"])
    d_b, _ = mocks.survey_catalogs(nd // 2, 1000, s["seed"] + 1000, **s["geo"])
    os.makedirs(workdir, exist_ok=True)
    cats, sums = {}, {}
    for key, cols in (("data_a", d_a), ("randoms_a", r_a), ("data_b", d_b)):
        cats[key] = mocks.write_fits_catalog(os.path.join(workdir, "c4_" + key + ".fits"), cols)
        sums[key] = float(sum(np.sum(v) for v in cols.values()))
    cats["randoms_b"] = cats["randoms_a"]
    return cats, sums


_BOX_CACHE = {}


def build_config_case(name, workdir):
    """Write the case's catalogs under ``workdir`` (once per catalog) and return
    (config, checksums)."""
    from cosmonpc_b200.mocks import lognormal_box

    over, cat = CONFIG_CASES[name]
    cfg = copy.deepcopy(over)
    cfg["output_dir"] = os.path.join(workdir, "out_" + name)
    if cat[0] == "survey":
        key = ("survey", workdir)
        if key not in _BOX_CACHE:
            _BOX_CACHE[key] = survey4_catalogs(workdir)
        cats, sums = _BOX_CACHE[key]
        cfg["catalogs"] = dict(cats)
        return cfg, dict(sums)
    _, npart, L, seed = cat
    key = (npart, L, seed, workdir)
    if key not in _BOX_CACHE:
        pos = lognormal_box(npart, L, seed)
        os.makedirs(workdir, exist_ok=True)
        path = os.path.join(workdir, "cat_%d_%d.npy" % (seed, npart))
        np.save(path, pos)
        _BOX_CACHE[key] = (path, {"a": float(np.sum(pos)), "n_a": float(len(pos))})
    path, sums = _BOX_CACHE[key]
    cfg["catalogs"] = {"data_a": path, "randoms_a": None, "data_b": None, "randoms_b": None}
    return cfg, dict(sums)
