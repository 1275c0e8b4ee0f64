"""Config validation with the reference's exact rules, exception types and
messages (src/cosmonpc/param_helper.py:1-165), so that a config rejected by the
reference is rejected here the same way."""
from __future__ import annotations

import numpy as np


def validate_tracer(tracer_type, correlation_mode):
    """param_helper.py:4-16."""
    assert correlation_mode in ["auto", "cross"], "correlation_mode must be either 'auto' or 'cross'"
    assert tracer_type in ["aaa", "aab", "abb", "abc"], \
        "tracer_type must be one of 'aaa', 'aab', 'abb', or 'abc'"
    if correlation_mode == "auto":
        assert tracer_type == "aaa", "For auto-correlation, tracer_type must be 'aaa'"


def validate_poles(poles):
    """param_helper.py:19-34."""
    if not all(isinstance(p, int) and p >= 0 for p in poles):
        raise ValueError("All elements in 'poles' must be non-negative integers.")
    if len(poles) != len(set(poles)):
        raise ValueError("'poles' contains duplicate values.")
    if len(poles) > 1 and poles != sorted(poles):
        raise ValueError("'poles' must be sorted in ascending order if it contains more than one value.")


def validate_sugi_poles(angu_config, geometry):
    """param_helper.py:37-59."""
    ell1, ell2, L = angu_config
    if ell1 < ell2:
        raise ValueError("In 'angu_config', ell1 must be greater than or equal to ell2.")
    if (ell1 + ell2 + L) % 2 != 0:
        raise ValueError("The sum of ell1, ell2, and L in 'angu_config' must be even.")
    if L % 2 != 0:
        raise ValueError("L must be even.")
    if not (ell1 - ell2 <= L <= ell1 + ell2):
        raise ValueError("The values in 'angu_config' do not satisfy the triangle condition.")
    if geometry not in ["box-like", "survey-like"]:
        raise ValueError("geometry must be either 'box-like' or 'survey-like'.")


def cubic_check(value, value_name, value_type):
    """param_helper.py:62-69 (Cubic_Check)."""
    assert isinstance(value, (list, tuple)) and len(value) == 3, \
        f"{value_name} must be a list or tuple of three elements"
    # The message reads value_type.__name__, so for a tuple of types (boxsize)
    # a failing element check raises AttributeError, exactly as the reference.
    assert all(isinstance(x, value_type) and x > 0 for x in value), \
        f"All elements in {value_name} must be positive {value_type.__name__}s"
    assert len(set(value)) == 1, f"All elements in {value_name} must be equal"


Cubic_Check = cubic_check


def validate_boolean_fields(config):
    """param_helper.py:72-87."""
    for field in ["interlaced", "compensation", "apply_rsd", "use_parent_dir"]:
        if field not in config:
            continue
        if not isinstance(config[field], (bool, np.bool_)):
            raise TypeError(
                f"Config field '{field}' must be a boolean (True/False), got "
                f"{type(config[field]).__name__}: {config[field]!r}")


def validate_config(config):
    """param_helper.py:90-136 (normalises aliases in place, like the reference)."""
    if "shotnoise-mode" in config and "shotnoise_mode" not in config:
        config["shotnoise_mode"] = config.pop("shotnoise-mode")
    if "high_order_mode" not in config:
        if "use_fast_mode" in config:
            config["high_order_mode"] = "fast" if config.pop("use_fast_mode") else "default"
        else:
            config["high_order_mode"] = "default"
    elif "use_fast_mode" in config:
        config.pop("use_fast_mode")
    assert config["sampler"] in ["ngp", "cic", "pcs", "tsc"], "sampler should be 'ngp', 'cic', 'pcs', or 'tsc'"
    cubic_check(config["nmesh"], "nmesh", int)
    cubic_check(config["boxsize"], "boxsize", (float, int))
    shotnoise_mode = config.setdefault("shotnoise_mode", "ana")
    if shotnoise_mode not in ["ana", "fft", "both"]:
        raise ValueError("shotnoise_mode must be either 'ana', 'fft', or 'both'")
    high_order_mode = config["high_order_mode"]
    if high_order_mode not in ["default", "fast", "compare"]:
        raise ValueError("high_order_mode must be one of 'default', 'fast', or 'compare'")
    if high_order_mode in ["fast", "compare"]:
        supported_poles = [[0, 2, 4], [0, 2, 4, 6], [0, 2, 4, 6, 8]]
        if config.get("statistic") != "pk" or config.get("geometry") != "survey-like":
            raise ValueError(
                "high_order_mode 'fast' and 'compare' are only supported for survey-like pk measurements")
        if config.get("correlation_mode") != "auto":
            raise ValueError("high_order_mode 'fast' and 'compare' are only supported for auto-correlation")
        if config.get("poles") not in supported_poles:
            raise ValueError(f"high_order_mode '{high_order_mode}' only supports poles {supported_poles}")
    validate_boolean_fields(config)


def catalog_check(catalogs, geometry, correlation_mode, statistic, tracer_type=None):
    """param_helper.py:139-165."""
    assert catalogs["data_a"] is not None, "data_a catalog must be provided"
    if statistic in ["pk", "bk_sco", "bk_sugi"]:
        if correlation_mode == "auto":
            if geometry == "survey-like":
                assert catalogs["randoms_a"] is not None, \
                    "randoms_a catalog must be provided for survey-like auto-correlation"
        elif correlation_mode == "cross":
            assert catalogs["data_b"] is not None, "data_b catalog must be provided for cross-correlation"
            if geometry == "survey-like":
                assert catalogs["randoms_a"] is not None, \
                    "randoms_a catalog must be provided for survey-like cross-correlation"
                assert catalogs["randoms_b"] is not None, \
                    "randoms_b catalog must be provided for survey-like cross-correlation"
    if tracer_type == "abc" and statistic in ["bk_sco", "bk_sugi"]:
        assert catalogs.get("data_c") is not None, \
            "data_c catalog must be provided for tracer_type 'abc' in bispectrum"
        if geometry == "survey-like":
            assert catalogs.get("randoms_c") is not None, \
                "randoms_c catalog must be provided for tracer_type 'abc' in survey-like bispectrum"
