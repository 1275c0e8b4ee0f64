"""Config-dict driver for the oracle's box path (no file output).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates the box branch
of ``run_task`` (src/cosmonpc/task_executor.py:11-328) and ``get_mesh_box``
(src/cosmonpc/mesh_generator.py:15-169) far enough to turn a config dict into
the estimator's numeric result dict.
"""
from __future__ import annotations

import numpy as np

from . import box


def _efunc_flat(om0, z):
    """E(z) of astropy's FlatLambdaCDM(H0, Om0) (Tcmb0 = 0), its evaluation order."""
    zp1 = float(z) + 1.0
    return np.sqrt(zp1 ** 2 * ((0.0 * zp1 + om0) * zp1 + 0.0) + (1.0 - om0))


def read_box_catalog(path, column_names, apply_rsd=False, cosmology=None, redshift_box=None, los=None,
                     boxsize=None):
    """``catalog_reader`` box branches: ``.npy`` (catalog_processor.py:354-386),
    ``.fits`` and ``.h5``/``.hdf5`` (:388-445, h5_reader :16-88) with ``add_rsd``
    (:648-693) when ``apply_rsd``."""
    if str(path).lower().endswith(".fits"):
        from cosmonpc_b200.fits import open_table

        t = open_table(path)
        names = [c for c in column_names if c in t.colnames()]
        data = t.read_columns(names)
        pos = np.zeros((t.nrows, 3))
        for axes in (("X", "Y", "Z"), ("x", "y", "z")):
            if all(a in names for a in axes):
                pos = np.column_stack([data[a] for a in axes]).astype(np.float64)
                break
        if apply_rsd:
            vel = None
            for axes in (("VX", "VY", "VZ"), ("vx", "vy", "vz")):
                if all(a in names for a in axes):
                    vel = np.column_stack([data[a] for a in axes]).astype(np.float64)
                    break
            factor = (1 + redshift_box) / (_efunc_flat(cosmology["Omega0"], redshift_box) * 100)
            los_v = np.array(los)
            if np.linalg.norm(los_v) != 1:
                raise ValueError("LOS must be a 3d unit vector")
            pos += factor * los_v * vel
            pos = pos % np.asarray(boxsize, dtype=np.float64)[0]
        w = np.asarray(data["w"], dtype=np.float64) if "w" in names else np.ones(t.nrows)
        return pos, w
    if str(path).lower().endswith((".h5", ".hdf5")):
        # h5_reader (cp:16-88) gives every requested name a field, so the
        # columns are chosen from column_names itself
        from cosmonpc_b200.hdf5 import read_dataset

        col = {}
        for c in column_names:
            try:
                col[c] = np.asarray(read_dataset(path, c), dtype=np.float64)
            except KeyError:
                pass
        n = len(next(iter(col.values()))) if col else 0
        pos = np.zeros((n, 3))
        for axes in (("X", "Y", "Z"), ("x", "y", "z")):
            if all(a in column_names for a in axes):
                pos = np.column_stack([col[a] for a in axes])
                break
        if apply_rsd:
            vel = None
            for axes in (("VX", "VY", "VZ"), ("vx", "vy", "vz")):
                if all(a in column_names for a in axes):
                    vel = np.column_stack([col[a] for a in axes])
                    break
            factor = (1 + redshift_box) / (_efunc_flat(cosmology["Omega0"], redshift_box) * 100)
            los_v = np.array(los)
            if np.linalg.norm(los_v) != 1:
                raise ValueError("LOS must be a 3d unit vector")
            pos += factor * los_v * vel
            pos = pos % np.asarray(boxsize, dtype=np.float64)[0]
        w = col["w"] if "w" in column_names else np.ones(n)
        return pos, w
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
        pos, w = read_box_catalog(cats["data_" + t], cfg["column_names"], cfg.get("apply_rsd", False),
                                  cfg.get("cosmology"), cfg.get("redshift_box"), cfg.get("rsd"),
                                  cfg["boxsize"])
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
