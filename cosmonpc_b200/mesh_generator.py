"""Mesh builders: catalogs -> painted device meshes.

``get_mesh_box`` mirrors src/cosmonpc/mesh_generator.py:15-169: it reads up to
three tracers (``.npy`` on the host; ``.fits`` decoded, and shifted into
redshift space when ``apply_rsd``, on the device), computes N_gal, sum(w) and
NZ = sum(w)/V in FP64, and paints them (interlaced pair in one pass) into
device meshes.
"""
from __future__ import annotations

import numpy as np
import torch

from . import engine
from .catalog_processor import read_box


def catalog_to_device(pos, w, pin=True):
    """Host arrays -> device tensors (through pinned memory)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    tp = torch.from_numpy(np.ascontiguousarray(pos, dtype=np.float64))
    tw = None if w is None else torch.from_numpy(np.ascontiguousarray(w, dtype=np.float64))
    if pin:
        tp = tp.pin_memory()
        tw = None if tw is None else tw.pin_memory()
    dp = tp.to(dev, non_blocking=True)
    dw = None if tw is None else tw.to(dev, non_blocking=True)
    return dp, dw


def paint_catalog(pos, w, nmesh, boxsize, sampler, interlaced, precision="f64"):
    """Paint a host or device catalog; returns (PaintedMesh, N_gal, weight_sum)."""
    n_gal = int(pos.shape[0])
    if isinstance(pos, torch.Tensor):
        weight_sum = float(w.sum().item())
        dp, dw = pos, w
    else:
        weight_sum = float(np.sum(w))
        dp, dw = catalog_to_device(pos, w)
    pm = engine.paint(dp, dw, int(nmesh[0]), float(boxsize[0]), sampler, interlaced, precision,
                      sum_w=weight_sum)
    return pm, n_gal, weight_sum


def get_mesh_box(catalogs, correlation_mode, nmesh, geometry, boxsize, sampler, interlaced,
                 column_names, comm=None, statistic="pk", tracer_type="ab", apply_rsd=False,
                 para_cosmo=None, redshift_box=None, los=None, precision="f64"):
    """Box meshes and number densities (mesh_generator.py:15-169)."""
    Nmesh = np.array(nmesh)
    box = np.array(boxsize)
    letters = ["a"]
    if correlation_mode == "cross":
        letters.append("b")
    if tracer_type == "abc":
        letters.append("c")
    meshes = {}
    attrs = {}
    for t in letters:
        pos, w = read_box(catalogs["data_" + t], column_names, apply_rsd, para_cosmo, redshift_box, los,
                          boxsize)
        pm, n_gal, wsum = paint_catalog(pos, w, Nmesh, box, sampler, interlaced, precision)
        meshes[t] = pm
        attrs["N_gal_" + t] = n_gal
        attrs["NZ_" + t] = wsum / np.prod(box)
    mesh_attrs = {}
    if correlation_mode == "auto":
        mesh_attrs.update({"NZ_a": attrs["NZ_a"], "N_gal_a": attrs["N_gal_a"]})
    else:
        mesh_attrs.update({"NZ_a": attrs["NZ_a"], "NZ_b": attrs["NZ_b"],
                           "N_gal_a": attrs["N_gal_a"], "N_gal_b": attrs["N_gal_b"]})
    if tracer_type == "abc":
        mesh_attrs.update({"NZ_c": attrs["NZ_c"], "N_gal_c": attrs["N_gal_c"]})
    mesh_attrs.update({"interlaced": interlaced, "sampler": sampler})
    if statistic == "pk":
        return mesh_attrs, meshes["a"], meshes.get("b")
    return mesh_attrs, meshes["a"], meshes.get("b"), meshes.get("c")
