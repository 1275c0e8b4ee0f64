"""Import the unmodified reference package on one CPU process.

Used only by ``make_golden.py`` in a container that has the reference sources.
The reference imports ``mpi4py``, ``numexpr``, ``pmesh``, ``astropy``, ``fitsio``
and ``h5py``; none is installed here, so this module places stand-ins in
``sys.modules`` before the import:

* ``mpi4py.MPI``: a one-rank communicator whose reductions are identities.
* ``numexpr.evaluate``: evaluates the expression string with numpy in the
  caller's frame (the form ``sympy.lambdify(..., "numexpr")`` emits).
* ``pmesh.pm.ParticleMesh``: ``oracle.pmesh_lite`` (restated pmesh behaviour).
* ``astropy.cosmology.FlatLambdaCDM``: comoving distance by ``scipy.integrate.quad``
  (a vectorised 64-point Gauss-Legendre rule for large catalogs); ``Planck18``
  with its photon and massive-neutrino densities (``oracle/cosmology.py``).
* ``fitsio.FITS``: this repository's FITS binary-table reader (``cosmonpc_b200.fits``).
* ``h5py.File``: this repository's HDF5 reader (``cosmonpc_b200.hdf5``).
"""
from __future__ import annotations

import math
import os
import sys
import types

import numpy as np

REFERENCE_SRC = os.environ.get("COSMONPC_REFERENCE_SRC", "/root/reference/src")
_HERE = os.path.dirname(os.path.abspath(__file__))
_REPO = os.path.dirname(os.path.dirname(_HERE))


class _Comm:
    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def reduce(self, x, op=None, root=0):
        return x

    def allreduce(self, x, op=None):
        return x

    def bcast(self, x, root=0):
        return x

    def gather(self, x, root=0):
        return [x]

    def allgather(self, x):
        return [x]

    def Barrier(self):
        return None

    def barrier(self):
        return None

    def Allreduce(self, sendbuf, recvbuf, op=None):
        src = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
        dst = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
        np.copyto(np.asarray(dst), np.asarray(src))


def _install_mpi():
    mpi4py = types.ModuleType("mpi4py")
    MPI = types.ModuleType("mpi4py.MPI")
    MPI.COMM_WORLD = _Comm()
    MPI.SUM, MPI.MIN, MPI.MAX = "sum", "min", "max"
    MPI.DOUBLE = "double"

    class Request:
        @staticmethod
        def Waitall(reqs):
            return None

    MPI.Request = Request
    mpi4py.MPI = MPI
    sys.modules["mpi4py"] = mpi4py
    sys.modules["mpi4py.MPI"] = MPI


def _install_numexpr():
    ne = types.ModuleType("numexpr")
    ne.__version__ = "2.14.1"
    funcs = {n: getattr(np, n) for n in (
        "sqrt", "sin", "cos", "tan", "exp", "log", "abs", "real", "imag", "conj",
        "where", "arctan2", "arcsin", "arccos", "arctan", "sinh", "cosh", "tanh")}
    funcs["complex"] = lambda a, b: np.asarray(a) + 1j * np.asarray(b)

    def evaluate(ex, local_dict=None, global_dict=None, **kw):
        frame = sys._getframe(1)
        ns = dict(funcs)
        ns.update(frame.f_globals if global_dict is None else global_dict)
        ns.update(frame.f_locals if local_dict is None else local_dict)
        return eval(ex, {"__builtins__": {}}, ns)

    ne.evaluate = evaluate
    sys.modules["numexpr"] = ne


def _install_pmesh():
    sys.path.insert(0, _REPO)
    from oracle import pmesh_lite

    pmesh = types.ModuleType("pmesh")
    pm = types.ModuleType("pmesh.pm")
    pm.ParticleMesh = pmesh_lite.ParticleMesh
    pm.RealField = pmesh_lite.RealField
    pm.ComplexField = pmesh_lite.ComplexField
    pm.TransposedComplexField = pmesh_lite.ComplexField
    pmesh.ParticleMesh = pmesh_lite.ParticleMesh
    pmesh.pm = pm
    sys.modules["pmesh"] = pmesh
    sys.modules["pmesh.pm"] = pm


def _install_astropy():
    from scipy.integrate import quad

    # the real astropy imports numpy.lib.recfunctions, which the reference's
    # add_completeness_weight reaches as np.lib.recfunctions
    import numpy.lib.recfunctions  # noqa: F401

    astropy = types.ModuleType("astropy")
    cosmo = types.ModuleType("astropy.cosmology")
    units = types.ModuleType("astropy.units")

    class _Q(float):
        @property
        def value(self):
            return float(self)

        def to(self, unit):
            return self

    class FlatLambdaCDM:
        def __init__(self, H0=70.0, Om0=0.3, Tcmb0=0.0, **kw):
            self.H0 = _Q(float(getattr(H0, "value", H0)))
            self.Om0 = float(Om0)
            self.h = self.H0 / 100.0

        def efunc(self, z):
            # astropy's evaluation order for a flat cosmology without radiation
            zp1 = np.asarray(z, dtype=np.float64) + 1.0
            return np.sqrt(zp1 ** 2 * ((0.0 * zp1 + self.Om0) * zp1 + 0.0) + (1.0 - self.Om0))

        def comoving_distance(self, z):
            # (c / H0) int_0^z dt / E(t).  Few redshifts: scipy quad per value;
            # large catalogs: t = z u with a 64-point Gauss-Legendre rule on
            # u in [0, 1] (E is analytic and smooth there, so both agree to
            # rounding), vectorised in chunks.
            c = 299792.458
            zz = np.atleast_1d(np.asarray(z, dtype=np.float64)).ravel()
            if zz.size <= 4096:
                out = np.array([quad(lambda t: 1.0 / float(self.efunc(t)), 0.0, zi)[0] for zi in zz])
            else:
                x, wt = np.polynomial.legendre.leggauss(64)
                u, wu = 0.5 * (x + 1.0), 0.5 * wt
                out = np.empty_like(zz)
                for i in range(0, zz.size, 65536):
                    zc = zz[i:i + 65536]
                    out[i:i + 65536] = zc * ((1.0 / self.efunc(zc[:, None] * u[None, :])) @ wu)
            out *= c / self.H0
            return _Arr(out.reshape(np.shape(z)))

    class _Arr(np.ndarray):
        def __new__(cls, a):
            return np.asarray(a).view(cls)

        @property
        def value(self):
            return np.asarray(self)

    class _Planck18(FlatLambdaCDM):
        """astropy's Planck18 realisation: photons and one massive neutrino
        (oracle/cosmology.py restates its background)."""

        def __init__(self):
            super().__init__(H0=67.66, Om0=0.30966)

        def efunc(self, z):
            from oracle import cosmology as oc

            return oc.efunc(z)

    cosmo.FlatLambdaCDM = FlatLambdaCDM
    cosmo.Planck18 = _Planck18()
    units.Mpc = 1.0
    units.km = 1.0
    units.s = 1.0
    astropy.cosmology = cosmo
    astropy.units = units
    sys.modules["astropy"] = astropy
    sys.modules["astropy.cosmology"] = cosmo
    sys.modules["astropy.units"] = units


def _install_fitsio():
    """``fitsio.FITS`` over this repository's FITS binary-table reader."""
    sys.path.insert(0, _REPO)
    from cosmonpc_b200 import fits as _fits

    fitsio = types.ModuleType("fitsio")

    class _HDU:
        def __init__(self, table):
            self._t = table

        def get_nrows(self):
            return self._t.nrows

        def get_colnames(self):
            return self._t.colnames()

        def read(self, rows=None, columns=None):
            cols = self._t.colnames() if columns is None else list(columns)
            sel = None if rows is None else np.asarray(list(rows), dtype=np.int64)
            return self._t.read_columns(cols, rows=sel)

    class FITS:
        def __init__(self, path, mode="r"):
            self._path = path
            self._n = len(_fits.hdu_list(path))

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def __len__(self):
            return self._n

        def __getitem__(self, i):
            return _HDU(_fits.open_table(self._path))

    fitsio.FITS = FITS
    sys.modules["fitsio"] = fitsio


def _install_h5py():
    """``h5py.File`` over this repository's HDF5 reader (root-group datasets)."""
    sys.path.insert(0, _REPO)
    from cosmonpc_b200 import hdf5 as _h5

    h5py = types.ModuleType("h5py")

    class _Dataset:
        def __init__(self, path, info):
            self._path, self._info, self._arr = path, info, None

        def __len__(self):
            return self._info.n

        def __getitem__(self, sl):
            if self._arr is None:
                self._arr = _h5.read_dataset(self._path, self._info.name)
            return self._arr[sl]

    class File:
        def __init__(self, path, mode="r"):
            self._path = path
            self._infos, _ = _h5.open_datasets(path)

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

        def __contains__(self, key):
            return key in self._infos

        def __getitem__(self, key):
            return _Dataset(self._path, self._infos[key])

        def keys(self):
            return list(self._infos)

    h5py.File = File
    sys.modules["h5py"] = h5py


def _install_placeholders():
    for name in ("fitsio", "h5py"):
        sys.modules.setdefault(name, types.ModuleType(name))


def import_reference():
    """Install the stand-ins and return the reference's ``cosmonpc`` package."""
    _install_mpi()
    _install_numexpr()
    _install_pmesh()
    _install_astropy()
    _install_fitsio()
    _install_h5py()
    _install_placeholders()
    if REFERENCE_SRC not in sys.path:
        sys.path.insert(0, REFERENCE_SRC)
    import cosmonpc  # noqa: F401  (the reference package)
    import cosmonpc.task_executor as te

    return te
