"""Catalog readers feeding the device path.

Box ``.npy`` catalogs: a memory-mapped (N, ncol) float array whose columns are
named by ``column_names``; ``x, y, z`` give the position and ``w`` (optional)
the weight (src/cosmonpc/catalog_processor.py:91-125, :354-386).  One process
reads the whole file (the reference splits rows over MPI ranks and reduces
the counts; the totals are identical).

Box ``.fits`` and ``.h5``/``.hdf5`` catalogs (src/cosmonpc/catalog_processor.py:
16-88, :388-445): positions from X, Y, Z or else x, y, z; velocities from VX,
VY, VZ or else vx, vy, vz when ``apply_rsd``; weight ``w``.  The raw columns go
to the device as stored and ``cnpc_box_catalog`` decodes them and applies the
redshift-space shift of add_rsd (catalog_processor.py:648-693).
"""
from __future__ import annotations

import math

import numpy as np

SUPPORTED = {"npy", "fits", "h5", "hdf5"}


def _ext(path):
    if isinstance(path, list):
        return path[0].split(".")[-1].lower() if path and path[0] else None
    return path.split(".")[-1].lower() if path else None


def flat_lcdm_efunc(omega_m, z):
    """E(z) of a flat LCDM cosmology without radiation, evaluated in the order
    astropy's FlatLambdaCDM(H0, Om0) uses (Tcmb0 = 0, so no photons or
    neutrinos): sqrt(zp1^2 ((0 zp1 + Om0) zp1 + 0) + Ode0), Ode0 = 1 - Om0."""
    zp1 = float(z) + 1.0
    ode0 = 1.0 - float(omega_m)
    return math.sqrt(zp1 ** 2 * ((0.0 * zp1 + float(omega_m)) * zp1 + 0.0) + ode0)


def rsd_shift(cosmology, redshift_box, los):
    """rsd_factor * los of add_rsd (catalog_processor.py:648-693, box branch):
    rsd_factor = (1 + z) / (100 E(z)) in (Mpc/h)/(km/s); the reference rejects
    a line of sight whose norm is not exactly 1."""
    e = flat_lcdm_efunc(cosmology["Omega0"], redshift_box)
    factor = (1 + redshift_box) / (e * 100)
    los = np.array(los)
    if np.linalg.norm(los) != 1:
        raise ValueError("LOS must be a 3d unit vector")
    return factor * los


def _pick(names, groups):
    for axes in groups:
        if all(a in names for a in axes):
            return axes
    return None


def read_box_fits(paths, column_names, apply_rsd=False, cosmology=None, redshift_box=None, los=None,
                  boxsize=None):
    """Box FITS catalog(s) decoded on the device: (positions (N, 3), weights (N,))
    as float64 CUDA tensors (files of a list concatenated in order)."""
    import torch

    from . import _lib
    from .fits import open_table

    paths = [paths] if isinstance(paths, str) else list(paths)
    tables = [open_table(p) for p in paths]
    names = [c for c in column_names if c in tables[0].colnames()] if tables else []
    pos_axes = _pick(names, [("X", "Y", "Z"), ("x", "y", "z")])
    vel_axes = _pick(names, [("VX", "VY", "VZ"), ("vx", "vy", "vz")]) if apply_rsd else None
    shift = None
    if apply_rsd:
        if vel_axes is None:
            # the reference reaches add_rsd with its velocity variable unset
            raise UnboundLocalError("cannot access local variable 'velocities' where it is not associated "
                                    "with a value")
        shift = rsd_shift(cosmology, redshift_box, los)
    box_length = float(np.asarray(boxsize, dtype=np.float64).reshape(-1)[0]) if boxsize is not None else 0.0
    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = _lib.Context.get()
    outs_p, outs_w = [], []
    for t in tables:
        raw = t.rows()
        host = torch.empty(raw.size, dtype=torch.uint8, pin_memory=True)
        if raw.size:
            np.copyto(host.numpy().reshape(raw.shape), raw)
        rows = host.to(dev, non_blocking=True)
        base = rows.data_ptr()

        def ref(name):
            if name is None:
                return _lib.ColRef(None, 0, _lib.CT_ABSENT, 0, 1.0, 0.0)
            c = t.scalar_column(name)
            if c.code not in _lib.CT_OF_FITS:
                raise ValueError(f"column {name}: unsupported FITS type {c.code}")
            return _lib.ColRef(base + c.offset, t.row_bytes, _lib.CT_OF_FITS[c.code], 1, c.scale, c.zero)

        cols = [ref(pos_axes[d] if pos_axes else None) for d in range(3)]
        cols += [ref(vel_axes[d] if vel_axes else None) for d in range(3)]
        cols.append(ref("w" if "w" in names else None))
        pos = torch.empty((max(t.nrows, 1), 3), dtype=torch.float64, device=dev)[:t.nrows]
        w = torch.empty(max(t.nrows, 1), dtype=torch.float64, device=dev)[:t.nrows]
        ctx.box_catalog(t.nrows, cols, apply_rsd, shift, box_length, pos, w)
        rows.record_stream(torch.cuda.current_stream(dev))
        outs_p.append(pos)
        outs_w.append(w)
    if len(outs_p) == 1:
        return outs_p[0], outs_w[0]
    return torch.cat(outs_p), torch.cat(outs_w)


def read_box(path, column_names, apply_rsd=False, cosmology=None, redshift_box=None, los=None, boxsize=None):
    """Box branch of catalog_reader (catalog_processor.py:354-445): ``.npy``
    catalogs as host arrays (the reference applies no RSD to them), ``.fits``
    catalogs decoded and shifted on the device."""
    ext = _ext(path)
    if ext not in SUPPORTED:
        raise ValueError(f"Unsupported data file type: {ext}")
    if ext == "npy":
        return read_box_npy(path, column_names)
    if ext == "fits":
        return read_box_fits(path, column_names, apply_rsd, cosmology, redshift_box, los, boxsize)
    return read_box_hdf5(path, column_names, apply_rsd, cosmology, redshift_box, los, boxsize)


_CT_OF_NUMPY = {"f8": "F64", "f4": "F32", "i8": "I64", "i4": "I32", "i2": "I16", "u1": "U8"}


def read_box_hdf5(paths, column_names, apply_rsd=False, cosmology=None, redshift_box=None, los=None,
                  boxsize=None):
    """Box HDF5 catalog(s) (h5_reader, catalog_processor.py:16-88, with the box
    branch :388-445) decoded, and shifted into redshift space, on the device.

    The reference builds its table with a field for every requested name, so
    the position, velocity and weight columns are chosen from ``column_names``
    itself; a chosen column that is not a dataset of the file would be left
    uninitialised there and raises ValueError here.  Contiguous datasets are
    copied to the device as stored; chunked (filtered) ones are inflated on the
    host first."""
    import torch

    from . import _lib
    from .hdf5 import _materialise, open_datasets

    paths = [paths] if isinstance(paths, str) else list(paths)
    names = list(column_names)
    pos_axes = _pick(names, [("X", "Y", "Z"), ("x", "y", "z")])
    vel_axes = _pick(names, [("VX", "VY", "VZ"), ("vx", "vy", "vz")]) if apply_rsd else None
    shift = None
    if apply_rsd:
        if vel_axes is None:
            raise UnboundLocalError("cannot access local variable 'velocities' where it is not associated "
                                    "with a value")
        shift = rsd_shift(cosmology, redshift_box, los)
    box_length = float(np.asarray(boxsize, dtype=np.float64).reshape(-1)[0]) if boxsize is not None else 0.0
    wanted = list(pos_axes or ()) + list(vel_axes or ()) + (["w"] if "w" in names else [])
    dev = torch.device("cuda", torch.cuda.current_device())
    ctx = _lib.Context.get()
    outs_p, outs_w = [], []
    for path in paths:
        infos, f = open_datasets(path)
        nrows = next((infos[c].n for c in names if c in infos), 0)
        keep = []  # device copies, alive until the decode is queued

        def ref(name):
            if name is None:
                return _lib.ColRef(None, 0, _lib.CT_ABSENT, 0, 1.0, 0.0)
            if name not in infos:
                raise ValueError(f"{path}: column {name} is not a dataset of the file")
            d = infos[name]
            if d.n != nrows:
                raise ValueError(f"{path}: dataset {name} has {d.n} rows, not {nrows}")
            code = _CT_OF_NUMPY.get(d.dtype.str[1:])
            if code is None:
                raise ValueError(f"{path}: dataset {name}: unsupported element type {d.dtype}")
            host = np.ascontiguousarray(_materialise(d, f))
            t = torch.from_numpy(host.view(np.uint8).copy()).pin_memory().to(dev, non_blocking=True)
            keep.append(t)
            return _lib.ColRef(t.data_ptr(), d.dtype.itemsize, getattr(_lib, "CT_" + code),
                               1 if d.dtype.byteorder == ">" else 0, 1.0, 0.0)

        cols = [ref(pos_axes[k] if pos_axes else None) for k in range(3)]
        cols += [ref(vel_axes[k] if vel_axes else None) for k in range(3)]
        cols.append(ref("w" if "w" in wanted else None))
        pos = torch.empty((max(nrows, 1), 3), dtype=torch.float64, device=dev)[:nrows]
        w = torch.empty(max(nrows, 1), dtype=torch.float64, device=dev)[:nrows]
        ctx.box_catalog(nrows, cols, apply_rsd, shift, box_length, pos, w)
        for t in keep:
            t.record_stream(torch.cuda.current_stream(dev))
        outs_p.append(pos)
        outs_w.append(w)
    if len(outs_p) == 1:
        return outs_p[0], outs_w[0]
    return torch.cat(outs_p), torch.cat(outs_w)


def read_box_npy(path, column_names):
    """Return (positions (N,3) float64, weights (N,) float64) of a box catalog."""
    ext = _ext(path)
    if ext not in SUPPORTED:
        raise ValueError(f"Unsupported data file type: {ext}")
    if ext != "npy":
        raise ValueError("read_box_npy reads .npy catalogs")
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
