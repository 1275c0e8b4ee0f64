"""Config-dict driver for the oracle's box path (no file output).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates the box branch
of ``run_task`` (src/cosmonpc/task_executor.py:11-328) and ``get_mesh_box``
(src/cosmonpc/mesh_generator.py:15-169) far enough to turn a config dict into
the estimator's numeric result dict.
"""
from __future__ import annotations

import numpy as np

from . import box


def read_box_catalog(path, column_names):
    """``catalog_reader`` box ``.npy`` branch (catalog_processor.py:354-386)."""
    arr = np.load(path, mmap_mode="r")
    idx = [column_names.index(a) for a in ("x", "y", "z")]
    pos = np.column_stack([arr[:, i] for i in idx]).astype(np.float64)
    if "w" in column_names:
        w = np.asarray(arr[:, column_names.index("w")], dtype=np.float64)
    else:
        w = np.ones(len(arr))
    return pos, w


def run_box(config):
    cfg = dict(config)
    n = int(cfg["nmesh"][0])
    L = float(cfg["boxsize"][0])
    V = L ** 3
    cats = cfg["catalogs"]
    mode = cfg["correlation_mode"]
    tracer = cfg.get("tracer_type", "ab")
    letters = ["a"]
    if mode == "cross":
        letters.append("b")
    if tracer == "abc":
        letters.append("c")
    fields, N_gal, NZ = {}, {}, {}
    for t in letters:
        pos, w = read_box_catalog(cats["data_" + t], cfg["column_names"])
        N_gal[t] = w.shape[0]
        NZ[t] = np.sum(w) / V
        fields[t] = box.paint_field(pos, w, n, L, cfg["sampler"], cfg["interlaced"])
    if cfg["statistic"] == "pk":
        return box.pk_box(fields["a"], fields.get("b"), mode, n, L, cfg["k_min"], cfg["k_max"],
                          cfg["k_bins"], cfg["poles"], cfg["sampler"], cfg["interlaced"],
                          cfg["rsd"], NZ["a"], NZ.get("b"))
    return box.bk_sugi_box(fields["a"], fields.get("b"), fields.get("c"), mode, tracer, n, L,
                           cfg["k_min"], cfg["k_max"], cfg["k_bins"], list(cfg["angu_config"]),
                           cfg["sampler"], cfg.get("data_vector_mode", "diagonal"),
                           cfg.get("shotnoise_mode", "ana"), N_gal, NZ)
