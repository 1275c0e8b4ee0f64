"""ctypes binding of libcosmonpc_b200.so (include/cosmonpc_b200.h).

There is no CPU fallback: if the shared library is missing, or no CUDA device is
present, importing or calling the device path raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from .angular import Harmonic

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcosmonpc_b200.so")

CNPC_OK, CNPC_EINVAL, CNPC_ENOMEM, CNPC_ECUDA, CNPC_ECUFFT, CNPC_ETIMEOUT = range(6)
F32, F64 = 0, 1
COMP_NONE, COMP_SINC, COMP_SHOTNOISE, COMP_BKNOISE = range(4)
WINDOW = {"ngp": 1, "cic": 2, "tsc": 3, "pcs": 4}

EXPORTED = (
    "cnpc_ctx_create", "cnpc_ctx_destroy", "cnpc_ctx_last_error", "cnpc_status_string",
    "cnpc_version", "cnpc_paint", "cnpc_fft_r2c", "cnpc_fft_c2r", "cnpc_forward_finish",
    "cnpc_kbin_counts", "cnpc_pk_bins", "cnpc_sn_bins", "cnpc_shell_spectra",
    "cnpc_contract_gram", "cnpc_contract_gram_noalloc",
)


class CnpcError(RuntimeError):
    """A CUDA / cuFFT failure reported by the library."""


class ShellItem(ctypes.Structure):
    """Mirror of ``cnpc_shell_item``."""

    _fields_ = [("bin", ctypes.c_int), ("harmonic", ctypes.c_int), ("component", ctypes.c_int),
                ("source", ctypes.c_int), ("conj", ctypes.c_int)]


_vp = ctypes.c_void_p
_i = ctypes.c_int
_i64 = ctypes.c_int64
_d = ctypes.c_double
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

_SIGS = {
    "cnpc_ctx_create": [ctypes.POINTER(_vp), _i],
    "cnpc_ctx_destroy": [_vp],
    "cnpc_ctx_last_error": [_vp],
    "cnpc_status_string": [_i],
    "cnpc_version": [],
    "cnpc_paint": [_vp, _i, _vp, _vp, _i64, _i, _d, _i, _vp, _vp, _vp],
    "cnpc_fft_r2c": [_vp, _i, _i, _i, _vp, _i64, _vp, _vp],
    "cnpc_fft_c2r": [_vp, _i, _i, _i, _vp, _vp, _i64, _vp],
    "cnpc_forward_finish": [_vp, _i, _i, _d, _vp, _vp, _d, _i, _i, _d, _d, _vp],
    "cnpc_kbin_counts": [_vp, _i, _d, _dp, _i, _vp, _vp, _vp],
    "cnpc_pk_bins": [_vp, _i, _i, _d, _vp, _vp, _dp, _i, _ip, _i, _dp, _vp, _vp],
    "cnpc_sn_bins": [_vp, _i, _i, _d, _vp, _vp, _d, _d, _i, ctypes.POINTER(Harmonic), _dp, _i,
                     _vp, _vp, _d, _vp],
    "cnpc_shell_spectra": [_vp, _i, _i, _d, _vp, _vp, _dp, _i, ctypes.POINTER(Harmonic), _i,
                           ctypes.POINTER(ShellItem), _i, _vp, _vp],
    "cnpc_contract_gram": [_vp, _i, _i64, _vp, _vp, _i64, _ip, _i, _ip, _i, _vp, _vp],
    "cnpc_contract_gram_noalloc": [_i, _i64, _vp, _vp, _i64, _ip, _i, _ip, _i, _vp, _vp],
}

_lib = None
_lock = threading.Lock()


def load():
    """Load the shared library (raises ImportError if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError("libcosmonpc_b200.so is not built (python -m cosmonpc_b200.build)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_char_p if name in ("cnpc_ctx_last_error", "cnpc_status_string") else _i
        _lib = lib
        return lib


def _darr(values):
    a = np.ascontiguousarray(values, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _iarr(values):
    a = np.ascontiguousarray(values, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


# kernels each entry point launches (cuFFT's own kernels are not counted)
KERNELS_PER_CALL = {"paint": 1, "forward_finish": 1, "kbin_counts": 1, "pk_bins": 1, "sn_bins": 1,
                    "shell_spectra": 1, "gram": 2}
launch_count = 0


def _count(name):
    global launch_count
    launch_count += KERNELS_PER_CALL.get(name, 0)


class KernelTimer:
    """Brackets every library call with CUDA events on the launching stream and
    records its algorithmic bytes (used by bench.py for live roofline numbers)."""

    def __init__(self):
        self.records = []

    def start(self):
        import torch

        e = torch.cuda.Event(enable_timing=True)
        e.record()
        return e

    def stop(self, name, e0, nbytes):
        import torch

        e1 = torch.cuda.Event(enable_timing=True)
        e1.record()
        self.records.append((name, e0, e1, nbytes))

    def summary(self):
        """{name: (launches, total_ms, total_bytes)} -- call after synchronising."""
        out = {}
        for name, e0, e1, nb in self.records:
            c, t, b = out.get(name, (0, 0.0, 0))
            out[name] = (c + 1, t + e0.elapsed_time(e1), b + nb)
        return out


timer = None


def _tstart():
    return timer.start() if timer is not None else None


def _tstop(name, e0, nbytes):
    if timer is not None:
        timer.stop(name, e0, nbytes)


def _esz(dtype):
    return 4 if dtype == F32 else 8


class Context:
    """One library context (cuFFT plan cache + scratch) per CUDA device."""

    _per_device = {}

    def __init__(self, device):
        self.lib = load()
        self.device = device
        h = _vp()
        st = self.lib.cnpc_ctx_create(ctypes.byref(h), device)
        if st != CNPC_OK:
            raise CnpcError("cnpc_ctx_create(%d) failed: %s" % (device, self.lib.cnpc_status_string(st).decode()))
        self.h = h

    @classmethod
    def get(cls, device=None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("cosmonpc_b200 needs a CUDA device; none is available")
        dev = torch.cuda.current_device() if device is None else int(device)
        ctx = cls._per_device.get(dev)
        if ctx is None:
            with torch.cuda.device(dev):
                ctx = cls(dev)
            cls._per_device[dev] = ctx
        return ctx

    def close(self):
        if self.h:
            self.lib.cnpc_ctx_destroy(self.h)
            self.h = None

    # ----------------------------------------------------------- helpers
    def _check(self, st, what):
        if st == CNPC_OK:
            return
        msg = self.lib.cnpc_ctx_last_error(self.h).decode() or self.lib.cnpc_status_string(st).decode()
        if st == CNPC_EINVAL:
            raise ValueError("%s: %s" % (what, msg))
        if st == CNPC_ENOMEM:
            raise MemoryError("%s: %s" % (what, msg))
        raise CnpcError("%s: %s" % (what, msg))

    @staticmethod
    def stream():
        import torch

        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    # ------------------------------------------------------------ calls
    def paint(self, dtype, pos, weight, n, boxsize, window, mesh, mesh_shifted):
        e0 = _tstart()
        st = self.lib.cnpc_paint(self.h, dtype, _ptr(pos), _ptr(weight), pos.shape[0], n, boxsize,
                                 window, _ptr(mesh), _ptr(mesh_shifted), self.stream())
        self._check(st, "cnpc_paint")
        _count("paint")
        _tstop("paint", e0, pos.shape[0] * (24 + (8 if weight is not None else 0))
               + n ** 3 * _esz(dtype) * (2 if mesh_shifted is not None else 1))

    def r2c(self, dtype, n, batch, real, spec, real_dist=0):
        e0 = _tstart()
        self._check(self.lib.cnpc_fft_r2c(self.h, dtype, n, batch, _ptr(real), real_dist, _ptr(spec), self.stream()),
                    "cnpc_fft_r2c")
        _tstop("cufft_r2c", e0, batch * (n ** 3 + 2 * n * n * (n // 2 + 1)) * _esz(dtype))

    def c2r(self, dtype, n, batch, spec, real, real_dist=0):
        e0 = _tstart()
        self._check(self.lib.cnpc_fft_c2r(self.h, dtype, n, batch, _ptr(spec), _ptr(real), real_dist, self.stream()),
                    "cnpc_fft_c2r")
        _tstop("cufft_c2r", e0, batch * (n ** 3 + 2 * n * n * (n // 2 + 1)) * _esz(dtype))

    def forward_finish(self, dtype, n, boxsize, spec, spec2, scale, comp, window, k0, band=0.0):
        e0 = _tstart()
        st = self.lib.cnpc_forward_finish(self.h, dtype, n, boxsize, _ptr(spec), _ptr(spec2), scale,
                                          comp, window, k0, band, self.stream())
        self._check(st, "cnpc_forward_finish")
        _count("forward_finish")
        _tstop("forward_finish", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * (3 if spec2 is not None else 2))

    def kbin_counts(self, n, boxsize, edges, counts, ksum):
        e, ep = _darr(edges)
        e0 = _tstart()
        st = self.lib.cnpc_kbin_counts(self.h, n, boxsize, ep, len(e), _ptr(counts), _ptr(ksum), self.stream())
        self._check(st, "cnpc_kbin_counts")
        _count("kbin_counts")
        _tstop("kbin_counts", e0, 0)

    def pk_bins(self, dtype, n, boxsize, a, b, edges, poles, los, sums):
        e, ep = _darr(edges)
        p, pp = _iarr(poles)
        l, lp = _darr(los)
        e0 = _tstart()
        st = self.lib.cnpc_pk_bins(self.h, dtype, n, boxsize, _ptr(a), _ptr(b), ep, len(e), pp, len(p),
                                   lp, _ptr(sums), self.stream())
        self._check(st, "cnpc_pk_bins")
        _count("pk_bins")
        _tstop("pk_bins", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * (1 if a.data_ptr() == b.data_ptr() else 2))

    def sn_bins(self, dtype, n, boxsize, a, b, vsq, sn0, window, yl0, edges, sums, source=None, band=0.0):
        e, ep = _darr(edges)
        yp = ctypes.byref(yl0) if yl0 is not None else None
        e0 = _tstart()
        st = self.lib.cnpc_sn_bins(self.h, dtype, n, boxsize, _ptr(a), _ptr(b), vsq, sn0, window, yp,
                                   ep, len(e), _ptr(sums), _ptr(source), band, self.stream())
        self._check(st, "cnpc_sn_bins")
        _count("sn_bins")
        _tstop("sn_bins", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype)
               * ((1 if a.data_ptr() == b.data_ptr() else 2) + (1 if source is not None else 0)))

    def shell_spectra(self, dtype, n, boxsize, a, b, edges, harmonics, items, out):
        e, ep = _darr(edges)
        harr = (Harmonic * len(harmonics))(*harmonics)
        iarr = (ShellItem * len(items))(*items)
        e0 = _tstart()
        st = self.lib.cnpc_shell_spectra(self.h, dtype, n, boxsize, _ptr(a), _ptr(b), ep, len(e), harr,
                                         len(harmonics), iarr, len(items), _ptr(out), self.stream())
        self._check(st, "cnpc_shell_spectra")
        _count("shell_spectra")
        nsrc = len({it.source for it in items if it.source < 2})
        _tstop("shell_spectra", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * (len(items) + nsrc))

    def gram(self, dtype, ncell, g, fields, stride, a_idx, b_idx, out):
        a, ap = _iarr(a_idx)
        b, bp = _iarr(b_idx)
        e0 = _tstart()
        st = self.lib.cnpc_contract_gram(self.h, dtype, ncell, _ptr(g), _ptr(fields), stride, ap, len(a),
                                         bp, len(b), _ptr(out), self.stream())
        self._check(st, "cnpc_contract_gram")
        _count("gram")
        _tstop("gram", e0, (len(set(a_idx) | set(b_idx)) + 1) * ncell * _esz(dtype))
        # (FP32 launches run on the tensor cores: gram_mma_kernel)
