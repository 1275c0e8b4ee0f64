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
    "cnpc_contract_gram", "cnpc_contract_gram_noalloc", "cnpc_paint_ex", "cnpc_catalog_decode",
    "cnpc_particle_sums", "cnpc_catalog_weights", "cnpc_interlace_split", "cnpc_xspace_harmonic",
    "cnpc_survey_bins", "cnpc_survey_source", "cnpc_field_product_sum", "cnpc_field_axpby",
    "cnpc_field_parity_fold",
    "cnpc_survey_hermitian_accumulate", "cnpc_shell_fields", "cnpc_contract_pairs",
    "cnpc_contract_gram_tc", "cnpc_contract_gram_multi_g", "cnpc_sn_bins_multi",
    "cnpc_forward_finish_band", "cnpc_ctx_set_wait_limit", "cnpc_ctx_take_status",
    "cnpc_contract_gram_tc_multi_g", "cnpc_box_catalog",
)

# survey catalog columns (cnpc_colid) and column types (cnpc_coltype)
COL_RA, COL_DEC, COL_Z, COL_WEIGHT, COL_SYSTOT, COL_NOZ, COL_CP, COL_FKP, COL_NZ, NCOLS = range(10)
CT_ABSENT, CT_F64, CT_F32, CT_I16, CT_I32, CT_I64, CT_U8, CT_BOOL = range(8)
CT_OF_FITS = {"D": CT_F64, "E": CT_F32, "I": CT_I16, "J": CT_I32, "K": CT_I64, "B": CT_U8, "L": CT_BOOL}
W_COLUMN, W_ONE, W_BOSS, W_EBOSS = range(4)
COSMO_FLAT_LCDM, COSMO_PLANCK18 = range(2)
PSUM_COUNT = 5


class CnpcError(RuntimeError):
    """A CUDA / cuFFT failure reported by the library."""


class DeviceTimeout(CnpcError):
    """A bounded device-side wait gave up (CNPC_ETIMEOUT): the outputs of the
    call that waited are NaN and the context stays usable."""


class ShellItem(ctypes.Structure):
    """Mirror of ``cnpc_shell_item``."""

    _fields_ = [("bin", ctypes.c_int), ("harmonic", ctypes.c_int), ("component", ctypes.c_int),
                ("source", ctypes.c_int), ("conj", ctypes.c_int)]


class Column(ctypes.Structure):
    """Mirror of ``cnpc_column``."""

    _fields_ = [("type", ctypes.c_int), ("offset", ctypes.c_int), ("scale", ctypes.c_double),
                ("zero", ctypes.c_double)]


class CatalogSpec(ctypes.Structure):
    """Mirror of ``cnpc_catalog_spec``."""

    _fields_ = [("row_bytes", ctypes.c_int64), ("col", Column * 9), ("weight_rule", ctypes.c_int),
                ("has_zrange", ctypes.c_int), ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
                ("h", ctypes.c_double), ("omega_m", ctypes.c_double), ("cosmology", ctypes.c_int)]


class ColRef(ctypes.Structure):
    """Mirror of ``cnpc_colref``."""

    _fields_ = [("d_base", ctypes.c_void_p), ("stride", ctypes.c_int64), ("type", ctypes.c_int),
                ("big_endian", ctypes.c_int), ("scale", ctypes.c_double), ("zero", ctypes.c_double)]


BOX_X, BOX_Y, BOX_Z, BOX_VX, BOX_VY, BOX_VZ, BOX_W, BOX_NCOLS = range(8)


class Operand(ctypes.Structure):
    """Mirror of ``cnpc_operand``."""

    _fields_ = [("p", ctypes.c_void_p), ("q", ctypes.c_void_p), ("scale", ctypes.c_double),
                ("comp", ctypes.c_int)]


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
    "cnpc_forward_finish_band": [_vp, _i, _i, _d, _vp, _vp, _d, _i, _i, _d, _d, _vp, _d, _vp],
    "cnpc_kbin_counts": [_vp, _i, _d, _dp, _i, _vp, _vp, _vp],
    "cnpc_pk_bins": [_vp, _i, _i, _d, _vp, _vp, _dp, _i, _ip, _i, _dp, _vp, _vp],
    "cnpc_sn_bins": [_vp, _i, _i, _d, _vp, _vp, _d, _d, _i, ctypes.POINTER(Harmonic), _dp, _i,
                     _vp, _vp, _d, _vp],
    "cnpc_sn_bins_multi": [_vp, _i, _i, _d, _vp, _vp, _d, _i, _i, _dp, ctypes.POINTER(ctypes.POINTER(Harmonic)),
                           _dp, _i, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _d, _vp],
    "cnpc_shell_spectra": [_vp, _i, _i, _d, _vp, _vp, _dp, _i, ctypes.POINTER(Harmonic), _i,
                           ctypes.POINTER(ShellItem), _i, _vp, _vp],
    "cnpc_contract_gram": [_vp, _i, _i64, _vp, _vp, _i64, _ip, _i, _ip, _i, _vp, _vp],
    "cnpc_contract_gram_noalloc": [_i, _i64, _vp, _vp, _i64, _ip, _i, _ip, _i, _vp, _vp],
    "cnpc_paint_ex": [_vp, _i, _vp, _vp, _i64, _i, _d, _i, _dp, _d, _i, _vp, _vp, _vp],
    "cnpc_catalog_decode": [_vp, _vp, _i64, ctypes.POINTER(CatalogSpec), _vp, _vp, _vp, _vp,
                            ctypes.POINTER(_i64), _vp],
    "cnpc_particle_sums": [_vp, _i64, _vp, _vp, _vp, _vp, ctypes.POINTER(Harmonic), _i, _vp, _vp],
    "cnpc_catalog_weights": [_vp, _i64, _vp, _vp, _i, _vp, _vp],
    "cnpc_interlace_split": [_vp, _i, _i, _d, _vp, _vp, _d, _i, _vp, _vp, _vp],
    "cnpc_xspace_harmonic": [_vp, _i, _i, _d, _dp, _vp, _vp, ctypes.POINTER(Harmonic), _i, _d, _vp, _vp,
                             _vp],
    "cnpc_survey_bins": [_vp, _i, _i, _d, _i, ctypes.POINTER(Operand), ctypes.POINTER(Operand), _d, _d,
                         ctypes.POINTER(Harmonic), _i, _d, _dp, _i, _vp, _vp],
    "cnpc_survey_source": [_vp, _i, _i, _d, _i, ctypes.POINTER(Operand), ctypes.POINTER(Operand), _d, _d,
                           _d, _vp, _vp, _vp],
    "cnpc_field_product_sum": [_vp, _i, _i64, _i, ctypes.POINTER(_vp), ctypes.POINTER(_vp), _vp, _vp],
    "cnpc_field_axpby": [_vp, _i, _i64, _d, _vp, _d, _vp, _vp, _vp],
    "cnpc_field_parity_fold": [_vp, _i, _i, _vp, _i, _vp, _vp],
    "cnpc_survey_hermitian_accumulate": [_vp, _i, _i, _d, _i, ctypes.POINTER(Operand),
                                         ctypes.POINTER(Harmonic), _d, _vp, _vp],
    "cnpc_shell_fields": [_vp, _i, _d, _vp, _vp, _dp, _i, ctypes.POINTER(Harmonic), _i,
                          ctypes.POINTER(ShellItem), _i, ctypes.POINTER(_vp), _vp],
    "cnpc_contract_pairs": [_vp, _i, _i64, _vp, _vp, _i64, _ip, _ip, _i, _vp, _vp],
    "cnpc_contract_gram_tc": [_vp, _i64, _vp, _vp, _i64, _ip, _i, _ip, _i, _vp, _vp],
    "cnpc_contract_gram_multi_g": [_vp, _i64, ctypes.POINTER(_vp), _i, _vp, _i64, _ip, _ip, _i, _ip, _i, _vp,
                                   _vp],
    "cnpc_contract_gram_tc_multi_g": [_vp, _i64, ctypes.POINTER(_vp), _i, _vp, _i64, _ip, _ip, _i, _ip, _i, _vp,
                                      _vp],
    "cnpc_box_catalog": [_vp, _i64, ctypes.POINTER(ColRef), _i, _dp, _d, _vp, _vp, _vp],
    "cnpc_ctx_set_wait_limit": [_vp, _i64],
    "cnpc_ctx_take_status": [_vp, _vp, _ip],
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
                    "shell_spectra": 1, "gram": 2, "catalog_decode": 3, "particle_sums": 2,
                    "catalog_weights": 1, "interlace_split": 1, "xspace_harmonic": 1, "survey_bins": 1,
                    "survey_source": 1, "field_product_sum": 2, "field_axpby": 1,
                    "hermitian_accumulate": 1, "shell_fields": 2, "contract_pairs": 3,
                    "gram_tc": 2, "gram_multi_g": 2, "sn_bins_multi": 1, "forward_finish_band": 1,
                    "box_catalog": 1, "field_parity_fold": 1}
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
    """One library context (cuFFT plan cache + scratch) per CUDA device and
    stream: work queued on the default stream (and CUDA graph captures) uses the
    device's primary context, every other stream gets its own, so data vectors
    queued on different streams can run concurrently without sharing scratch."""

    _per_device = {}

    def __init__(self, device):
        self.lib = load()
        self.device = device
        h = _vp()
        st = self.lib.cnpc_ctx_create(ctypes.byref(h), device)
        if st != CNPC_OK:
            raise CnpcError("cnpc_ctx_create(%d) failed: %s" % (device, self.lib.cnpc_status_string(st).decode()))
        self.h = h

    _override = []  # contexts pinned by context_scope (innermost last)

    @classmethod
    def get(cls, device=None):
        import torch

        if cls._override and device is None:
            return cls._override[-1]
        if not torch.cuda.is_available():
            raise RuntimeError("cosmonpc_b200 needs a CUDA device; none is available")
        dev = torch.cuda.current_device() if device is None else int(device)
        key = dev
        if not torch.cuda.is_current_stream_capturing():
            s = torch.cuda.current_stream(dev).cuda_stream
            if s != torch.cuda.default_stream(dev).cuda_stream:
                key = (dev, s)
        ctx = cls._per_device.get(key)
        if ctx is None:
            with torch.cuda.device(dev):
                ctx = cls(dev)
            cls._per_device[key] = ctx
        return ctx

    @classmethod
    def scope(cls, ctx):
        """Within ``with Context.scope(ctx):`` every call uses ``ctx`` (a CUDA
        graph captured inside keeps that context's workspaces)."""
        import contextlib

        @contextlib.contextmanager
        def _scope():
            cls._override.append(ctx)
            try:
                yield ctx
            finally:
                cls._override.pop()

        return _scope()

    def close(self):
        if self.h:
            self.lib.cnpc_ctx_destroy(self.h)
            self.h = None

    @classmethod
    def release_all(cls):
        """Destroy every cached context (plans, workspaces) after synchronising
        the device; later calls create fresh ones."""
        import torch

        torch.cuda.synchronize()
        for ctx in list(cls._per_device.values()):
            ctx.close()
        cls._per_device.clear()

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

    def box_catalog(self, nrows, cols, apply_rsd, shift, box_length, pos, weight):
        """cnpc_box_catalog: ``cols`` is a list of BOX_NCOLS ColRef."""
        arr = (ColRef * BOX_NCOLS)(*cols)
        sh, shp = _darr(shift if shift is not None else (0.0, 0.0, 0.0))
        st = self.lib.cnpc_box_catalog(self.h, int(nrows), arr, 1 if apply_rsd else 0, shp, float(box_length),
                                       _ptr(pos), _ptr(weight), self.stream())
        self._check(st, "cnpc_box_catalog")
        _count("box_catalog")

    def set_wait_limit(self, polls):
        """Polls a bounded device wait makes before it gives up (0: at once)."""
        self._check(self.lib.cnpc_ctx_set_wait_limit(self.h, int(polls)), "cnpc_ctx_set_wait_limit")

    def take_status(self, stream=None):
        """Synchronise ``stream`` (a torch stream; default: the current one), read
        and clear this context's device status word; raises DeviceTimeout if a
        bounded wait gave up since the last read."""
        v = ctypes.c_int(0)
        sh = self.stream() if stream is None else ctypes.c_void_p(stream.cuda_stream)
        self._check(self.lib.cnpc_ctx_take_status(self.h, sh, ctypes.byref(v)), "cnpc_ctx_take_status")
        if v.value == CNPC_ETIMEOUT:
            raise DeviceTimeout("a bounded device wait gave up (CNPC_ETIMEOUT); the results of the call are NaN")
        if v.value != CNPC_OK:
            raise CnpcError("device status word %d" % v.value)

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

    def forward_finish_band(self, dtype, n, boxsize, spec, spec2, scale, comp, window, k0, band, band_out,
                            band_out_k):
        e0 = _tstart()
        st = self.lib.cnpc_forward_finish_band(self.h, dtype, n, boxsize, _ptr(spec), _ptr(spec2), scale,
                                               comp, window, k0, band, _ptr(band_out), band_out_k, self.stream())
        self._check(st, "cnpc_forward_finish_band")
        _count("forward_finish_band")
        _tstop("forward_finish", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * (4 if spec2 is not None else 3))

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

    def sn_bins_multi(self, dtype, n, boxsize, a, b, vsq, window, sn0s, yl0s, edges, sums, sources, band=0.0):
        """cnpc_sn_bins_multi: len(sn0s) (1 or 2) configurations in one pass;
        yl0s[c] / sources[c] may be None."""
        nc = len(sn0s)
        e, ep = _darr(edges)
        s0 = (ctypes.c_double * nc)(*[float(x) for x in sn0s])
        ys = (ctypes.POINTER(Harmonic) * nc)(*[ctypes.pointer(y) if y is not None else None for y in yl0s])
        ds = (_vp * nc)(*[t.data_ptr() for t in sums])
        ss = (_vp * nc)(*[t.data_ptr() if t is not None else None for t in sources])
        e0 = _tstart()
        st = self.lib.cnpc_sn_bins_multi(self.h, dtype, n, boxsize, _ptr(a), _ptr(b), vsq, window, nc, s0, ys,
                                         ep, len(e), ds, ss, band, self.stream())
        self._check(st, "cnpc_sn_bins_multi")
        _count("sn_bins_multi")
        _tstop("sn_bins", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype)
               * ((1 if a.data_ptr() == b.data_ptr() else 2) + sum(1 for x in sources if x is not None)))

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

    def shell_fields(self, n, boxsize, a, b, edges, harmonics, items, outs):
        """Fused synthesis + band-limited inverse FFT of FP32 shell fields."""
        e, ep = _darr(edges)
        harr = (Harmonic * len(harmonics))(*harmonics)
        iarr = (ShellItem * len(items))(*items)
        optr = (_vp * len(outs))(*[_ptr(t) for t in outs])
        e0 = _tstart()
        st = self.lib.cnpc_shell_fields(self.h, n, boxsize, _ptr(a), _ptr(b), ep, len(e), harr, len(harmonics),
                                        iarr, len(items), optr, self.stream())
        self._check(st, "cnpc_shell_fields")
        _count("shell_fields")
        nsrc = len({it.source for it in items if it.source < 2})
        # algorithmic: band of each source read once, each field written once
        band = n * (n // 2) * (n // 4) * 8
        _tstop("shell_fields", e0, len(items) * n ** 3 * 4 + nsrc * band // 2)

    def gram(self, dtype, ncell, g, fields, stride, a_idx, b_idx, out):
        a, ap = _iarr(a_idx)
        b, bp = _iarr(b_idx)
        e0 = _tstart()
        st = self.lib.cnpc_contract_gram(self.h, dtype, ncell, _ptr(g), _ptr(fields), stride, ap, len(a),
                                         bp, len(b), _ptr(out), self.stream())
        self._check(st, "cnpc_contract_gram")
        _count("gram")
        _tstop("gram", e0, (len(set(a_idx) | set(b_idx)) + 1) * ncell * _esz(dtype))

    def gram_tc(self, ncell, g, fields, stride, a_idx, b_idx, out):
        a, ap = _iarr(a_idx)
        b, bp = _iarr(b_idx)
        e0 = _tstart()
        st = self.lib.cnpc_contract_gram_tc(self.h, ncell, _ptr(g), _ptr(fields), stride, ap, len(a), bp, len(b),
                                            _ptr(out), self.stream())
        self._check(st, "cnpc_contract_gram_tc")
        _count("gram_tc")
        _tstop("gram", e0, (len(set(a_idx) | set(b_idx)) + 1) * ncell * 4)

    def gram_tc_multi_g(self, ncell, gs, fields, stride, a_idx, a_g, b_idx, out):
        """Tensor-core FP32 Gram whose row i is weighted by gs[a_g[i]] (one launch)."""
        a, ap = _iarr(a_idx)
        ag, agp = _iarr(a_g)
        b, bp = _iarr(b_idx)
        garr = (_vp * len(gs))(*[_ptr(t) for t in gs])
        e0 = _tstart()
        st = self.lib.cnpc_contract_gram_tc_multi_g(self.h, ncell, garr, len(gs), _ptr(fields), stride, ap, agp,
                                                    len(a), bp, len(b), _ptr(out), self.stream())
        self._check(st, "cnpc_contract_gram_tc_multi_g")
        _count("gram_tc")
        _tstop("gram", e0, (len(set(a_idx) | set(b_idx)) + len(gs)) * ncell * 4)

    def gram_multi_g(self, ncell, gs, fields, stride, a_idx, a_g, b_idx, out):
        """FP32 Gram whose row i is weighted by gs[a_g[i]] (one launch)."""
        a, ap = _iarr(a_idx)
        ag, agp = _iarr(a_g)
        b, bp = _iarr(b_idx)
        garr = (_vp * len(gs))(*[_ptr(t) for t in gs])
        e0 = _tstart()
        st = self.lib.cnpc_contract_gram_multi_g(self.h, ncell, garr, len(gs), _ptr(fields), stride, ap, agp, len(a),
                                                 bp, len(b), _ptr(out), self.stream())
        self._check(st, "cnpc_contract_gram_multi_g")
        _count("gram_multi_g")
        _tstop("gram", e0, (len(set(a_idx) | set(b_idx)) + len(gs)) * ncell * 4)

    def contract_pairs(self, dtype, ncell, g, fields, stride, a_idx, b_idx, out):
        a, ap = _iarr(a_idx)
        b, bp = _iarr(b_idx)
        e0 = _tstart()
        st = self.lib.cnpc_contract_pairs(self.h, dtype, ncell, _ptr(g), _ptr(fields), stride, ap, bp, len(a),
                                          _ptr(out), self.stream())
        self._check(st, "cnpc_contract_pairs")
        _count("contract_pairs")
        _tstop("contract_pairs", e0, (len(set(a_idx) | set(b_idx)) + 1) * ncell * _esz(dtype))

    # ------------------------------------------------------ survey path
    def paint_ex(self, dtype, pos, weight, n, boxsize, window, origin, mass_scale, accumulate, mesh,
                 mesh_shifted):
        o, op = _darr(origin if origin is not None else [0.0, 0.0, 0.0])
        e0 = _tstart()
        st = self.lib.cnpc_paint_ex(self.h, dtype, _ptr(pos), _ptr(weight), pos.shape[0], n, boxsize,
                                    window, op, float(mass_scale), int(bool(accumulate)), _ptr(mesh),
                                    _ptr(mesh_shifted), self.stream())
        self._check(st, "cnpc_paint_ex")
        _count("paint")
        _tstop("paint", e0, pos.shape[0] * (24 + (8 if weight is not None else 0))
               + n ** 3 * _esz(dtype) * (2 if mesh_shifted is not None else 1))

    def catalog_decode(self, rows, nrows, spec, pos, w, wfkp, nz):
        kept = _i64(0)
        st = self.lib.cnpc_catalog_decode(self.h, _ptr(rows), nrows, ctypes.byref(spec), _ptr(pos), _ptr(w),
                                          _ptr(wfkp), _ptr(nz), ctypes.byref(kept), self.stream())
        self._check(st, "cnpc_catalog_decode")
        _count("catalog_decode")
        return int(kept.value)

    def particle_sums(self, np_, pos, w, wfkp, nz, harmonics, out):
        harr = (Harmonic * max(1, len(harmonics)))(*harmonics)
        st = self.lib.cnpc_particle_sums(self.h, np_, _ptr(pos), _ptr(w), _ptr(wfkp), _ptr(nz), harr,
                                         len(harmonics), _ptr(out), self.stream())
        self._check(st, "cnpc_particle_sums")
        _count("particle_sums")

    def catalog_weights(self, np_, w, wfkp, power, out):
        st = self.lib.cnpc_catalog_weights(self.h, np_, _ptr(w), _ptr(wfkp), power, _ptr(out), self.stream())
        self._check(st, "cnpc_catalog_weights")
        _count("catalog_weights")

    def interlace_split(self, dtype, n, boxsize, spec, spec2, scale, accumulate, herm, anti):
        e0 = _tstart()
        st = self.lib.cnpc_interlace_split(self.h, dtype, n, boxsize, _ptr(spec), _ptr(spec2), float(scale),
                                           int(bool(accumulate)), _ptr(herm), _ptr(anti), self.stream())
        self._check(st, "cnpc_interlace_split")
        _count("interlace_split")
        _tstop("interlace_split", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * 4)

    def xspace_harmonic(self, dtype, n, boxsize, boxcenter, re, im, harmonic, conj, scale, out_re, out_im):
        b, bp = _darr(boxcenter)
        e0 = _tstart()
        st = self.lib.cnpc_xspace_harmonic(self.h, dtype, n, boxsize, bp, _ptr(re), _ptr(im),
                                           ctypes.byref(harmonic), int(bool(conj)), float(scale), _ptr(out_re),
                                           _ptr(out_im), self.stream())
        self._check(st, "cnpc_xspace_harmonic")
        _count("xspace_harmonic")
        nio = 1 + (im is not None) + 1 + (out_im is not None)
        _tstop("xspace_harmonic", e0, n ** 3 * _esz(dtype) * nio)

    @staticmethod
    def operand(p, q=None, scale=1.0, comp=COMP_NONE):
        return Operand(_ptr(p), _ptr(q), float(scale), int(comp))

    def survey_bins(self, dtype, n, boxsize, window, u, v, sbar, harmonic, conj_z, weight, edges, sums):
        e, ep = _darr(edges)
        hp = ctypes.byref(harmonic) if harmonic is not None else None
        e0 = _tstart()
        st = self.lib.cnpc_survey_bins(self.h, dtype, n, boxsize, window, ctypes.byref(u), ctypes.byref(v),
                                       float(np.real(sbar)), float(np.imag(sbar)), hp, int(bool(conj_z)),
                                       float(weight), ep, len(e), _ptr(sums), self.stream())
        self._check(st, "cnpc_survey_bins")
        _count("survey_bins")
        nsp = 2 + (u.q is not None) + (v.q is not None)
        _tstop("survey_bins", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * nsp)

    def survey_source(self, dtype, n, boxsize, window, u, v, sbar, band, herm, anti):
        e0 = _tstart()
        st = self.lib.cnpc_survey_source(self.h, dtype, n, boxsize, window, ctypes.byref(u), ctypes.byref(v),
                                         float(np.real(sbar)), float(np.imag(sbar)), float(band), _ptr(herm),
                                         _ptr(anti), self.stream())
        self._check(st, "cnpc_survey_source")
        _count("survey_source")
        _tstop("survey_source", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * 5)

    def hermitian_accumulate(self, dtype, n, boxsize, window, x, harmonic, weight, out):
        e0 = _tstart()
        st = self.lib.cnpc_survey_hermitian_accumulate(self.h, dtype, n, boxsize, window, ctypes.byref(x),
                                                       ctypes.byref(harmonic), float(weight), _ptr(out),
                                                       self.stream())
        self._check(st, "cnpc_survey_hermitian_accumulate")
        _count("hermitian_accumulate")
        _tstop("hermitian_accumulate", e0, n * n * (n // 2 + 1) * 2 * _esz(dtype) * 4)

    def field_product_sum(self, dtype, ncell, res, ims, out):
        nf = len(res)
        ra = (_vp * nf)(*[_ptr(t) for t in res])
        ia = (_vp * nf)(*[_ptr(t) for t in ims])
        st = self.lib.cnpc_field_product_sum(self.h, dtype, ncell, nf, ra, ia, _ptr(out), self.stream())
        self._check(st, "cnpc_field_product_sum")
        _count("field_product_sum")

    def field_parity_fold(self, dtype, n, src, sign, out):
        """out[(n/2 + 1) n^2] = the parity fold of ``src`` (n^3) with ``sign``
        (cnpc_field_parity_fold)."""
        st = self.lib.cnpc_field_parity_fold(self.h, dtype, n, _ptr(src), int(sign), _ptr(out), self.stream())
        self._check(st, "cnpc_field_parity_fold")
        _count("field_parity_fold")

    def field_axpby(self, dtype, ncell, a, x, b, y, out):
        st = self.lib.cnpc_field_axpby(self.h, dtype, ncell, float(a), _ptr(x), float(b), _ptr(y), _ptr(out),
                                       self.stream())
        self._check(st, "cnpc_field_axpby")
        _count("field_axpby")
