"""In-memory entry points (no catalog files): one call turns a catalog held in
host or device memory into the reference's result dictionaries.

``bk_sugi_box_vector`` is the fast form: several angular configurations of one
catalog share the paint, the forward transforms, G, the shell fields and the
FFT shot-noise shells; fields are FP32 with FP64 accumulation.
``bk_sugi_box_plain`` is the plain drop-in form: FP64 throughout, one
configuration per call (as ``run_stats`` is called once per configuration).
"""
from __future__ import annotations

import numpy as np
import torch

from . import clustering_estimator as ce
from . import engine


_COPY_STREAMS = {}


def _h2d(host, dev):
    """Device copy of a host array on a side stream, so that it overlaps the
    work already queued on the current stream; the current stream waits for
    the copy before its next launch."""
    t = torch.from_numpy(np.ascontiguousarray(host, dtype=np.float64))
    if not t.is_pinned():
        t = t.pin_memory()
    cs = _COPY_STREAMS.get(dev.index)
    if cs is None:
        cs = _COPY_STREAMS[dev.index] = torch.cuda.Stream(dev)
    cur = torch.cuda.current_stream(dev)
    with torch.cuda.stream(cs):
        d = torch.empty(t.shape, dtype=t.dtype, device=dev)
        d.copy_(t, non_blocking=True)
    cur.wait_stream(cs)
    d.record_stream(cur)
    return d


def _to_device(pos, weight):
    dev = torch.device("cuda", torch.cuda.current_device())
    if isinstance(pos, np.ndarray):
        pos = _h2d(pos, dev)
    if isinstance(weight, np.ndarray):
        weight = _h2d(weight, dev)
    return pos, weight


def _weight_sum(pos, weight):
    if weight is None:
        return float(pos.shape[0])
    if isinstance(weight, np.ndarray):
        return float(np.sum(weight))
    return float(weight.sum().item())


def box_attrs(n_gal, weight_sum, box_length, **settings):
    """stat_attrs of an auto box run (mesh_generator.py:56-60, :106-117)."""
    attrs = dict(settings)
    attrs.update({"NZ_a": weight_sum / float(np.prod(np.array([box_length] * 3))), "N_gal_a": int(n_gal)})
    return attrs


def bk_sugi_box_vector(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins,
                       angu_configs, data_vector_mode="full", shotnoise_mode="both",
                       precision="f32", block_size="full", deferred=False):
    """Auto bispectrum multipoles of one box catalog for every configuration in
    ``angu_configs`` (list of (l1, l2, L)); returns a list of result dicts, or
    with ``deferred`` a function returning them once the device work of this
    catalog is enqueued (the next catalog's work can then be enqueued before
    this one's host algebra runs)."""
    wsum = _weight_sum(pos, weight)
    dpos, dw = _to_device(pos, weight)
    pm = engine.paint(dpos, dw, nmesh, boxsize, sampler, interlaced, precision, sum_w=wsum)
    attrs = box_attrs(dpos.shape[0], wsum, boxsize, boxsize=[boxsize] * 3, nmesh=[nmesh] * 3,
                      k_min=k_min, k_max=k_max, k_bins=k_bins, sampler=sampler, interlaced=interlaced,
                      data_vector_mode=data_vector_mode, shotnoise_mode=shotnoise_mode)
    finalize = ce.bk_sugi_box_submit({"a": pm}, "auto", "aaa", [tuple(c) for c in angu_configs], attrs,
                                     precision=precision, block_size=block_size)
    return finalize if deferred else finalize()


def bk_sugi_box_plain(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins,
                      angu_configs, data_vector_mode="full", shotnoise_mode="both", block_size="full"):
    """The plain FP64 drop-in: one full per-configuration call each, like
    repeated ``run_stats`` calls without the file I/O."""
    out = []
    for cfg in angu_configs:
        out += bk_sugi_box_vector(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins,
                                  [cfg], data_vector_mode, shotnoise_mode, precision="f64",
                                  block_size=block_size)
    return out


def pk_box_vector(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins, poles,
                  rsd=(0, 0, 1), precision="f32"):
    """Auto power-spectrum multipoles of one box catalog."""
    wsum = _weight_sum(pos, weight)
    dpos, dw = _to_device(pos, weight)
    pm = engine.paint(dpos, dw, nmesh, boxsize, sampler, interlaced, precision, sum_w=wsum)
    attrs = box_attrs(dpos.shape[0], wsum, boxsize, boxsize=[boxsize] * 3, nmesh=[nmesh] * 3,
                      k_min=k_min, k_max=k_max, k_bins=k_bins, sampler=sampler, interlaced=interlaced,
                      poles=list(poles), rsd=list(rsd))
    return ce.calculate_power_spectrum_box(pm, None, "auto", attrs)


def mock_pk_bk(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins, poles=(0, 2, 4),
               angu_configs=((0, 0, 0),), data_vector_mode="diagonal", shotnoise_mode="ana", precision="f32",
               rsd=(0, 0, 1), deferred=False, sum_w=None):
    """Power-spectrum multipoles and bispectrum configurations of one mock from a
    single paint: the interlaced R2C spectra are finished twice (the power
    spectrum and the bispectrum overdensity use different scalings and k = 0
    values).  Returns (pk result dict, [bk result dict per configuration]), or
    with ``deferred`` a function returning them, after the device work of this
    mock is queued, so that the next mock can be queued before the results are
    read.  ``sum_w``: the weight sum when it is known (no device read).  The
    deferred function takes an optional ``n_gal`` (and ``sn_unit``, see
    ``clustering_estimator.bk_sugi_box_submit``) for a catalog whose real count
    differs from the rows painted (zero-weight padding)."""
    wsum = _weight_sum(pos, weight) if sum_w is None else float(sum_w)
    dpos, dw = _to_device(pos, weight)
    pm = engine.paint(dpos, dw, nmesh, boxsize, sampler, interlaced, precision, sum_w=wsum)
    pm_bk = engine.PaintedMesh(pm.raw.clone(), pm.n, pm.boxsize, pm.sampler, pm.interlaced, pm.N_gal, pm.sum_w,
                               pm.precision)
    common = dict(boxsize=[boxsize] * 3, nmesh=[nmesh] * 3, k_min=k_min, k_max=k_max, k_bins=k_bins,
                  sampler=sampler, interlaced=interlaced)
    pk = ce.calculate_power_spectrum_box(pm, None, "auto", box_attrs(dpos.shape[0], wsum, boxsize,
                                                                      poles=list(poles), rsd=list(rsd), **common),
                                         deferred=True)
    attrs = box_attrs(dpos.shape[0], wsum, boxsize, data_vector_mode=data_vector_mode,
                      shotnoise_mode=shotnoise_mode, **common)
    bk = ce.bk_sugi_box_submit({"a": pm_bk}, "auto", "aaa", [tuple(c) for c in angu_configs], attrs,
                               precision=precision, block_size=None)
    volume = float(boxsize) ** 3

    def finalize(n_gal=None, sn_unit=None):
        if n_gal is None:
            return pk(), bk()
        return pk(NZ_a=float(n_gal) / volume), bk(n_gal=int(n_gal), sn_unit=sn_unit)

    return finalize if deferred else finalize()


class MockGraphs:
    """:func:`mock_pk_bk` for a stream of mocks of one shape class (mesh, box,
    settings) replayed from CUDA graphs: the device work of one mock (paint,
    transforms, shell fields, contractions, copies of the sums to pinned host
    memory) is captured once per slot and replayed for every mock, so the host
    no longer issues ~100 launches per mock.

    Catalogs may hold any number of particles up to ``capacity`` (no weights,
    inside the box): a slot's input is a ``capacity``-row catalog with
    per-particle weights; a catalog of N particles fills the first N rows with
    weight 1 and the rest with weight 0 at the origin, so the captured paint
    deposits exactly the catalog's mass.  The count enters only the host
    algebra (N_gal, the number density, the normalisation) and the analytic
    shot-noise sums, which are linear in the count and are moved from the
    captured one with the sums of a zero spectrum (``sn_unit``, computed once
    per class).  The FFT S3 term of (0,0,0) depends on the count through its
    source field, so with shotnoise_mode "fft"/"both" and (0,0,0) every catalog
    must have exactly ``capacity`` particles.

    ``submit(pos)`` copies ``pos`` into the slot's input, replays, and returns a
    function that waits for that replay and returns (pk result, [bk results]);
    call it before submitting ``slots`` more mocks.  Raises RuntimeError when
    the device work cannot be captured (then use :func:`mock_pk_bk`)."""

    def __init__(self, capacity, nmesh, boxsize, slots=2, **kw):
        from . import _lib

        self.kw = dict(kw, nmesh=nmesh, boxsize=boxsize)
        self.capacity = int(capacity)
        self.slots = []
        self.count = 0
        cfgs = [tuple(c) for c in kw.get("angu_configs", ((0, 0, 0),))]
        self.fixed_count = kw.get("shotnoise_mode", "ana") != "ana" and (0, 0, 0) in cfgs
        dev = torch.device("cuda", torch.cuda.current_device())
        self.sn_unit = self._sn_unit(dev)
        for _ in range(slots):
            # each slot: its own stream and library context, so replays of
            # different slots share no workspace and can overlap
            ctx = _lib.Context(dev.index)
            stream = torch.cuda.Stream(dev)
            pos = torch.empty((self.capacity, 3), dtype=torch.float64, device=dev)
            pos.uniform_(0.0, float(boxsize) * (1.0 - 1e-12))
            w = torch.ones(self.capacity, dtype=torch.float64, device=dev)
            stream.wait_stream(torch.cuda.current_stream(dev))
            with _lib.Context.scope(ctx):
                with torch.cuda.stream(stream):
                    for _ in range(2):  # plans, workspaces and pinned buffers at their final sizes
                        mock_pk_bk(pos, w, sum_w=self.capacity, **self.kw)
                stream.synchronize()
                graph = torch.cuda.CUDAGraph()
                try:
                    with torch.cuda.graph(graph, stream=stream, capture_error_mode="relaxed"):
                        fin = mock_pk_bk(pos, w, deferred=True, sum_w=self.capacity, **self.kw)
                except Exception as e:  # a host synchronisation or allocation inside the work
                    raise RuntimeError("mock pipeline could not be captured: %s" % e) from e
            self.slots.append((pos, w, graph, fin, stream, ctx))

    def _sn_unit(self, dev):
        """{L: k3-bin shot-noise sums of a zero spectrum with sn0 = 1} for the
        configurations whose sums depend on the count ((0,0,0) of an auto run)."""
        from . import _lib

        kw = self.kw
        if (0, 0, 0) not in [tuple(c) for c in kw.get("angu_configs", ((0, 0, 0),))]:
            return {}
        n, L = int(kw["nmesh"]), float(kw["boxsize"])
        precision = kw.get("precision", "f32")
        code, _, cdt = engine.PRECISION[precision]
        k_min, k_max, k_bins = kw["k_min"], kw["k_max"], kw["k_bins"]
        k3_edge = np.linspace(2 * k_min, 2 * k_max, k_bins * 2 + 1)[:-1]
        zero = torch.zeros((n, n, n // 2 + 1), dtype=cdt, device=dev)
        d = torch.empty(2 * (len(k3_edge) - 1), dtype=torch.float64, device=dev)
        _lib.Context.get().sn_bins(code, n, L, zero, zero, (L ** 3) ** 2, 1.0, _lib.WINDOW[kw["sampler"]], None,
                                   k3_edge, d)
        return {0: d.cpu().numpy()}

    def close(self):
        """Release the captured graphs, their memory pools and the slots' library
        contexts (cuFFT plans and workspaces)."""
        for (_, _, graph, _, stream, ctx) in self.slots:
            stream.synchronize()
            del graph
            ctx.close()
        self.slots = []

    def submit(self, pos):
        inp, w, graph, fin, stream, _ = self.slots[self.count % len(self.slots)]
        npart = int(pos.shape[0])
        if pos.ndim != 2 or pos.shape[1] != 3 or npart > self.capacity or npart < 1:
            raise ValueError("catalog of shape %s does not fit the captured capacity %d"
                             % (tuple(pos.shape), self.capacity))
        if self.fixed_count and npart != self.capacity:
            raise ValueError("with FFT shot noise of (0,0,0) every catalog needs exactly %d particles" % self.capacity)
        self.count += 1
        stream.wait_stream(torch.cuda.current_stream())  # pos was written on the caller's stream
        with torch.cuda.stream(stream):
            inp[:npart].copy_(pos, non_blocking=True)
            w[:npart].fill_(1.0)
            if npart < self.capacity:
                inp[npart:].zero_()
                w[npart:].zero_()
            graph.replay()
            done = torch.cuda.Event()
            done.record()
        pos.record_stream(stream)
        sn_unit = self.sn_unit

        def finalize():
            done.synchronize()
            return fin(n_gal=npart, sn_unit=sn_unit)

        return finalize


def mock_pk_bk_plain(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins, poles=(0, 2, 4),
                     angu_configs=((0, 0, 0),), data_vector_mode="diagonal", shotnoise_mode="ana", rsd=(0, 0, 1)):
    """The plain FP64 per-call form of :func:`mock_pk_bk`: one power-spectrum and
    one bispectrum call per mock, each painting its catalog (as separate
    ``run_stats`` calls do)."""
    pk = pk_box_vector(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins, poles, rsd,
                       precision="f64")
    bk = bk_sugi_box_plain(pos, weight, nmesh, boxsize, sampler, interlaced, k_min, k_max, k_bins, angu_configs,
                           data_vector_mode, shotnoise_mode, block_size=None)
    return pk, bk
