"""CPU restatement of the slice of the ``pmesh`` API that CosmoNPC's mesh path uses.

TEST INFRASTRUCTURE ONLY.  This module is part of the oracle: it is imported by
``tests/``, by ``tests/golden/make_golden.py`` (to run the unmodified reference
estimator code on CPU), by ``__graft_entry__.smoke()`` and by ``bench.py``'s CPU
baseline arm.  The product package never imports it.

pmesh (>= 0.1.59, ``pyproject.toml:17`` of the reference) is not vendored with the
reference and is not installed here, so its behaviour is restated from the
published algorithm and from how the reference uses it:

* ``ParticleMesh(BoxSize, Nmesh, dtype="complex128", resampler=...)``
  (``src/cosmonpc/mesh_generator.py:189-191``).  With a complex dtype every
  "real" field is a complex128 N^3 array and every transform is a full
  complex-to-complex FFT; ``r2c`` is normalised by 1/N^3 and ``c2r`` is not
  (the normalisation algebra of ``clustering_estimator.py:698-722`` relies on it).
* ``paint``: B-spline mass assignment of order p (NEAREST=1, CIC=2, TSC=3,
  PCS=4) onto nodes at integer grid coordinates ``i`` where the grid coordinate of
  a particle is ``g = x * Nmesh / BoxSize (+ shift)``; a node receives
  ``mass * prod_d W_p(i_d - g_d)``, periodic wrap (``mesh_generator.py:193-205``).
* ``affine.shift(0.5)``: the interlaced second paint at ``g + 0.5``
  (``mesh_generator.py:201-205``).
* ``ComplexField.x``: wave vectors ``k = n * 2 * pi / BoxSize`` with ``n`` in FFT
  order, the Nyquist index negative (``n = -N/2``); ``RealField.x``: node
  coordinates ``i * BoxSize / Nmesh`` wrapped into ``[-L/2, L/2)``
  (used by ``math_evaluator.py:12-32``).
* ``apply(func, kind="circular")``: calls ``func(w, v)`` with
  ``w_d = k_d * BoxSize_d / Nmesh_d`` in ``[-pi, pi)`` (``math_evaluator.py:206-309``).
* ``decompose`` / ``exchange``: identity on a single rank.

Because pmesh itself is absent, parity at this boundary is unpinned by any
reference test: the window node convention and k-vector formula above are the
published pmesh conventions restated, not measured.
"""
from __future__ import annotations

import numpy as np

try:  # scipy's pocketfft is multi-threaded; numpy's is the fallback.
    import scipy.fft as _fft

    def _fftn(a):
        return _fft.fftn(a, workers=-1)

    def _ifftn(a):
        return _fft.ifftn(a, workers=-1)

except Exception:  # pragma: no cover
    _fftn = np.fft.fftn
    _ifftn = np.fft.ifftn


WINDOW_SUPPORT = {"nearest": 1, "ngp": 1, "cic": 2, "tsc": 3, "pcs": 4}


def window_weights(s, order):
    """B-spline window W_p(s) of order p evaluated at offsets s (grid units)."""
    a = np.abs(s)
    if order == 1:
        return (a < 0.5).astype(np.float64)
    if order == 2:
        return np.where(a < 1.0, 1.0 - a, 0.0)
    if order == 3:
        return np.where(a < 0.5, 0.75 - a * a,
                        np.where(a < 1.5, 0.5 * (1.5 - a) ** 2, 0.0))
    if order == 4:
        return np.where(a < 1.0, (4.0 - 6.0 * a * a + 3.0 * a ** 3) / 6.0,
                        np.where(a < 2.0, (2.0 - a) ** 3 / 6.0, 0.0))
    raise ValueError(order)


def first_node(g, order):
    """Left-most node with non-zero weight for a particle at grid coordinate g."""
    if order % 2 == 0:
        return np.floor(g).astype(np.int64) - (order // 2 - 1)
    return np.floor(g + 0.5).astype(np.int64) - (order - 1) // 2


def paint_mass(grid_pos, mass, nmesh, order):
    """Deposit ``mass`` at grid coordinates ``grid_pos`` (Np,3) onto an N^3 mesh.

    Returns a float64 mesh.  Uses one ``bincount`` per window node offset so that
    10^6-particle catalogs paint in seconds.
    """
    n = np.asarray(nmesh, dtype=np.int64)
    g = np.asarray(grid_pos, dtype=np.float64)
    mass = np.broadcast_to(np.asarray(mass, dtype=np.float64), (g.shape[0],))
    base = [first_node(g[:, d], order) for d in range(3)]
    w1d = []
    idx1d = []
    for d in range(3):
        wd = []
        idd = []
        for o in range(order):
            node = base[d] + o
            wd.append(window_weights(node - g[:, d], order))
            idd.append(np.mod(node, n[d]))
        w1d.append(wd)
        idx1d.append(idd)
    out = np.zeros(int(n.prod()), dtype=np.float64)
    for ox in range(order):
        for oy in range(order):
            wxy = mass * w1d[0][ox] * w1d[1][oy]
            ixy = (idx1d[0][ox] * n[1] + idx1d[1][oy]) * n[2]
            for oz in range(order):
                flat = ixy + idx1d[2][oz]
                out += np.bincount(flat, weights=wxy * w1d[2][oz], minlength=out.size)
    return out.reshape(tuple(n))


class _Resampler:
    def __init__(self, name):
        key = name.lower()
        if key not in WINDOW_SUPPORT:
            raise ValueError("unknown resampler %s" % name)
        self.name = key
        self.support = WINDOW_SUPPORT[key]


class Affine:
    def __init__(self, scale, translate):
        self.scale = np.asarray(scale, dtype=np.float64)
        self.translate = np.asarray(translate, dtype=np.float64)

    def shift(self, amount):
        return Affine(self.scale, self.translate + amount)


class _Layout:
    def exchange(self, arr):
        return arr


class _Slabs:
    def __init__(self, field):
        self._field = field

    def __iter__(self):
        yield self._field

    @property
    def x(self):
        return [self._field.x]


class _Field(np.ndarray):
    def __new__(cls, pm, value):
        obj = np.asarray(value).view(cls)
        obj.pm = pm
        return obj

    def __array_finalize__(self, obj):
        self.pm = getattr(obj, "pm", None)

    @property
    def slabs(self):
        return _Slabs(self)

    @property
    def slices(self):
        return tuple(slice(0, int(n)) for n in self.pm.Nmesh)

    @property
    def cshape(self):
        return tuple(int(n) for n in self.pm.Nmesh)


class RealField(_Field):
    def r2c(self, out=None):
        n = float(np.prod(self.pm.Nmesh))
        return ComplexField(self.pm, _fftn(np.asarray(self, dtype=np.complex128)) / n)

    @property
    def x(self):
        return self.pm.x


class ComplexField(_Field):
    def c2r(self, out=None):
        n = float(np.prod(self.pm.Nmesh))
        return RealField(self.pm, _ifftn(np.asarray(self, dtype=np.complex128)) * n)

    @property
    def x(self):
        return self.pm.k

    def apply(self, func, kind="wavenumber", out=None):
        if kind == "circular":
            coords = self.pm.w
        elif kind == "wavenumber":
            coords = self.pm.k
        else:
            raise ValueError(kind)
        res = func(coords, np.asarray(self))
        if out is Ellipsis:
            self[...] = res
            return self
        if out is None:
            return ComplexField(self.pm, np.array(res, dtype=np.complex128))
        out[...] = res
        return out


class ParticleMesh:
    """Single-rank stand-in for ``pmesh.pm.ParticleMesh`` (see module docstring)."""

    def __init__(self, BoxSize, Nmesh, dtype="complex128", resampler="cic", comm=None):
        self.Nmesh = np.array(np.broadcast_to(np.asarray(Nmesh, dtype=np.int64), (3,)))
        self.BoxSize = np.array(np.broadcast_to(np.asarray(BoxSize, dtype=np.float64), (3,)))
        self.dtype = np.dtype(dtype)
        self.resampler = _Resampler(resampler)
        self.comm = comm
        self.affine = Affine(self.Nmesh / self.BoxSize, np.zeros(3))
        self.k = []
        self.w = []
        self.x = []
        for d in range(3):
            shape = [1, 1, 1]
            shape[d] = int(self.Nmesh[d])
            n = np.arange(self.Nmesh[d], dtype=np.int64)
            n[n >= self.Nmesh[d] // 2] -= self.Nmesh[d]
            k = n * 2 * np.pi / self.BoxSize[d]
            self.k.append(k.reshape(shape))
            self.w.append((k * (self.BoxSize[d] / self.Nmesh[d])).reshape(shape))
            xi = np.arange(self.Nmesh[d], dtype=np.float64) * self.BoxSize[d] / self.Nmesh[d]
            xi[xi >= 0.5 * self.BoxSize[d]] -= self.BoxSize[d]
            self.x.append(xi.reshape(shape))

    def decompose(self, pos, smoothing=0):
        return _Layout()

    def create(self, type="real", value=None):
        shape = tuple(int(n) for n in self.Nmesh)
        arr = np.zeros(shape, dtype=np.complex128)
        if value is not None:
            arr[...] = value
        return (RealField if type == "real" else ComplexField)(self, arr)

    def paint(self, position, mass=1.0, layout=None, transform=None, resampler=None, out=None):
        tr = self.affine if transform is None else transform
        pos = np.asarray(position, dtype=np.float64)
        g = pos * tr.scale + tr.translate
        order = (_Resampler(resampler) if resampler else self.resampler).support
        mesh = paint_mass(g, mass, self.Nmesh, order)
        return RealField(self, mesh.astype(np.complex128))
