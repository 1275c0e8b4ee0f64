"""``run_stats(config)`` -- the reference's public entry point
(src/cosmonpc/task_executor.py:11-343), same config keys, defaults,
validation errors, output file names and result dictionaries.

One process drives one GPU; ``comm`` arguments of the reference's internals are
accepted and ignored.  The optional config key ``precision`` selects the
arithmetic ("f64", default: the plain FP64 drop-in; "f32": FP32 fields with
FP64 accumulation).
"""
from __future__ import annotations

import logging
import os
import time

import numpy as np

from . import clustering_estimator as ce
from . import mesh_generator as mg
from .param_helper import (catalog_check, validate_config, validate_poles, validate_sugi_poles,
                           validate_tracer)

log = logging.getLogger("cosmonpc_b200")


def _save(output_dir, name, res):
    if not os.path.exists(output_dir):
        os.makedirs(output_dir)
    path = os.path.join(output_dir, name)
    np.save(path, res)
    return path


def run_task(statistic, correlation_mode, geometry, catalogs, **kwargs):
    """task_executor.py:11-328."""
    from . import survey

    survey.clear_cache()
    try:
        return _run_task(statistic, correlation_mode, geometry, catalogs, **kwargs)
    finally:
        survey.clear_cache()


def _run_task(statistic, correlation_mode, geometry, catalogs, **kwargs):
    k_max, nmesh, boxsize = kwargs["k_max"], kwargs["nmesh"], kwargs["boxsize"]
    nyquist_freq = np.pi * nmesh[0] / boxsize[0]
    precision = kwargs.get("precision", "f64")
    t0 = time.time()
    out_path = None

    if statistic == "pk":
        if k_max >= nyquist_freq:
            raise ValueError(
                f"k_max {k_max} is larger than the Nyquist frequency {nyquist_freq}. \
                                Please choose a smaller k_max.")
        validate_poles(kwargs["poles"])
        if geometry == "survey-like":
            from . import survey

            stat_attrs, rfield_a, rfield_b = survey.get_mesh_pk_survey(
                catalogs, correlation_mode, nmesh=nmesh, geometry=geometry,
                column_names=kwargs["column_names"], boxsize=boxsize, sampler=kwargs["sampler"],
                interlaced=kwargs["interlaced"], z_range=kwargs["z_range"],
                comp_weight_plan=kwargs["comp_weight_plan"], para_cosmo=kwargs["cosmology"],
                normalization_scheme=kwargs["normalization_scheme"],
                alpha_scheme=kwargs.get("alpha_scheme", "pypower"), precision=precision)
        else:
            poles = kwargs["poles"]
            if all(p % 2 == 1 for p in poles):
                raise ValueError(
                    f"All poles in {poles} are odd. Please choose at least one even pole, \
                                 since odd poles are defaultly set to 0 for periodic boxes.")
            stat_attrs, rfield_a, rfield_b = mg.get_mesh_box(
                catalogs, correlation_mode, nmesh=kwargs["nmesh"], geometry=geometry,
                boxsize=kwargs["boxsize"], sampler=kwargs["sampler"], interlaced=kwargs["interlaced"],
                column_names=kwargs["column_names"], statistic=statistic,
                apply_rsd=kwargs["apply_rsd"], para_cosmo=kwargs["cosmology"],
                redshift_box=kwargs["redshift_box"], los=kwargs["rsd"], precision=precision)
        stat_attrs.update(kwargs)
        stat_attrs["nyquist_freq"] = nyquist_freq
        t1 = time.time()
        if geometry == "survey-like":
            from . import survey

            pk_res = survey.calculate_power_spectrum_survey(stat_attrs, rfield_a, rfield_b,
                                                            correlation_mode, **kwargs)
        else:
            pk_res = ce.calculate_power_spectrum_box(rfield_a, rfield_b, correlation_mode,
                                                     stat_attrs, **kwargs)
        del rfield_a, rfield_b
        pk_res.update(stat_attrs)
        if geometry == "box-like":
            for key in ["z_range", "scheme"]:
                pk_res.pop(key, None)
        output_dir = kwargs.get("output_dir")
        name_a = os.path.splitext(os.path.basename(catalogs["data_a"]))[0]
        if correlation_mode == "auto":
            fname = f"pk_res_{correlation_mode}_{name_a}.npy"
        else:
            name_b = os.path.splitext(os.path.basename(catalogs["data_b"]))[0]
            fname = f"pk_res_{correlation_mode}_{name_a}_{name_b}.npy"
        out_path = _save(output_dir, fname, pk_res)
        log.info("power spectrum: %.2f s (fields %.2f s) -> %s", time.time() - t0, t1 - t0, out_path)

    if statistic == "bk_sugi":
        tracer_type = kwargs["tracer_type"]
        angu_config = kwargs["angu_config"]
        data_vector_mode = kwargs.get("data_vector_mode", "diagonal")
        shotnoise_mode = kwargs.get("shotnoise_mode", "ana")
        if data_vector_mode not in ["diagonal", "full"]:
            raise ValueError("data_vector_mode must be either 'diagonal' or 'full'")
        if shotnoise_mode not in ["ana", "fft", "both"]:
            raise ValueError("shotnoise_mode must be either 'ana', 'fft', or 'both'")
        if data_vector_mode == "diagonal":
            kwargs.setdefault("block_size", 1)
        else:
            kwargs.setdefault("block_size", "full")
        validate_tracer(tracer_type, correlation_mode)
        if 2 * k_max >= nyquist_freq:
            raise ValueError(
                f"2 * k_max = {2 * k_max} is larger than the Nyquist frequency {nyquist_freq}. \
                             Please choose a smaller k_max.")
        if geometry == "box-like":
            validate_sugi_poles(angu_config, geometry)
            stat_attrs, rfield_a, rfield_b, rfield_c = mg.get_mesh_box(
                catalogs, correlation_mode, statistic=statistic, nmesh=kwargs["nmesh"],
                geometry=geometry, boxsize=kwargs["boxsize"], sampler=kwargs["sampler"],
                interlaced=kwargs["interlaced"], column_names=kwargs["column_names"],
                tracer_type=tracer_type, apply_rsd=kwargs["apply_rsd"], para_cosmo=kwargs["cosmology"],
                redshift_box=kwargs["redshift_box"], los=kwargs["rsd"], precision=precision)
        else:
            validate_sugi_poles(angu_config, geometry)
            from . import survey

            stat_attrs, rfield_a, rfield_b, rfield_c = survey.get_mesh_bk_survey(
                catalogs, correlation_mode, tracer_type=tracer_type, angu_config=angu_config,
                nmesh=kwargs["nmesh"], geometry=geometry, column_names=kwargs["column_names"],
                boxsize=kwargs["boxsize"], sampler=kwargs["sampler"], interlaced=kwargs["interlaced"],
                z_range=kwargs["z_range"], comp_weight_plan=kwargs["comp_weight_plan"],
                para_cosmo=kwargs["cosmology"],
                normalization_scheme=kwargs.get("normalization_scheme", "particle"),
                alpha_scheme=kwargs.get("alpha_scheme", "pypower"), precision=precision)
        stat_attrs.update(kwargs)
        stat_attrs["nyquist_freq"] = nyquist_freq
        t1 = time.time()
        if geometry == "box-like":
            bk_res = ce.calculate_bk_sugi_box(rfield_a, rfield_b, rfield_c, correlation_mode,
                                              stat_attrs, **kwargs)
        else:
            from . import survey

            bk_res = survey.calculate_bk_sugi_survey(rfield_a, rfield_b, rfield_c, correlation_mode,
                                                     stat_attrs, catalogs=catalogs, **kwargs)
        bk_res.update(stat_attrs)
        if geometry == "box-like":
            keys_to_remove = ["z_range", "comp_weight_plan", "scheme", "alpha_scheme", "normalization_scheme"]
        else:
            keys_to_remove = ["redshift_box", "los", "apply_rsd"]
        for key in keys_to_remove:
            bk_res.pop(key, None)
        output_dir = kwargs.get("output_dir")
        name_a = os.path.splitext(os.path.basename(catalogs["data_a"]))[0]
        parent_dir = os.path.basename(os.path.dirname(catalogs["data_a"]))
        if kwargs.get("use_parent_dir", True):
            name_a = parent_dir + "_" + name_a
        fname = (f"bk_sugi_res_{data_vector_mode}_{angu_config[0]}{angu_config[1]}{angu_config[2]}"
                 f"_{correlation_mode}_{tracer_type}_{name_a}.npy")
        out_path = _save(output_dir, fname, bk_res)
        log.info("bispectrum: %.2f s (fields %.2f s) -> %s", time.time() - t0, t1 - t0, out_path)
    return out_path


def run_stats(config):
    """task_executor.py:330-343."""
    validate_config(config)
    catalog_check(config["catalogs"], config["geometry"], config["correlation_mode"], config["statistic"])
    os.makedirs(config["output_dir"], exist_ok=True)
    return run_task(**config)
