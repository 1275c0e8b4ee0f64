"""Catalog readers feeding the device path.

Box ``.npy`` catalogs: a memory-mapped (N, ncol) float array whose columns are
named by ``column_names``; ``x, y, z`` give the position and ``w`` (optional)
the weight (src/cosmonpc/catalog_processor.py:91-125, :354-386).  One process
reads the whole file (the reference splits rows over MPI ranks and reduces
the counts; the totals are identical).
"""
from __future__ import annotations

import numpy as np

SUPPORTED = {"npy", "fits", "h5", "hdf5"}


def _ext(path):
    if isinstance(path, list):
        return path[0].split(".")[-1].lower() if path and path[0] else None
    return path.split(".")[-1].lower() if path else None


def read_box_npy(path, column_names):
    """Return (positions (N,3) float64, weights (N,) float64) of a box catalog."""
    ext = _ext(path)
    if ext not in SUPPORTED:
        raise ValueError(f"Unsupported data file type: {ext}")
    if ext != "npy":
        raise NotImplementedError("box catalogs other than .npy are not supported by this build")
    assert column_names is not None and len(column_names) >= 3, (
        "For box-like geometry with .npy file, column_names must be provided "
        "with at least 3 elements for x,y,z.")
    arr = np.load(path, mmap_mode="r")
    idx = [column_names.index(axis) for axis in ["x", "y", "z"]]
    pos = np.empty((arr.shape[0], 3), dtype=np.float64)
    for d, i in enumerate(idx):
        pos[:, d] = arr[:, i]
    if "w" in column_names:
        w = np.ascontiguousarray(arr[:, column_names.index("w")], dtype=np.float64)
    else:
        w = np.ones(arr.shape[0], dtype=np.float64)
    return pos, w
