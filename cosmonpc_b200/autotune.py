"""Per-shape-class execution plans, measured once per device and cached on disk.

The reference leaves the memory/throughput trade-off of the bispectrum to its
``block_size`` setting (clustering_estimator.py:867-879, task_executor.py:
166-169): how many k-bins' shell fields are held at once.  Here that choice
and the batch depth of the shell-field synthesis are made per shape class:

* block size: the largest bin block whose shell fields fit the device-memory
  budget (80 % of the free HBM, ``engine.fields_capacity``), because a block
  of all bins computes every field once and smaller blocks recompute fields
  (the reference's own block loop); a requested ``block_size`` still caps it;
* shell items per synthesis call (``ShellFields.fft_batch``): the fused FP32
  band-limited kernels and the shell-spectra + cuFFT route both take a batch
  of fields per call; deeper batches fill the GPU better and cost one pass-1
  work array (fused) or one half spectrum (cuFFT) per field.  The candidates
  whose batch (with a cuFFT workspace of about its size) stays within 10 % of
  the device are timed on a synthetic spectrum of the class (CUDA events, best
  of a few repetitions, on a context of their own that is destroyed after, so
  the losing plans' workspaces are freed); a depth whose plan cannot be made is
  skipped, and the deepest batch within 2 % of the fastest per field wins
  (depths that close are run-to-run noise apart; deeper means fewer launches).

Plans are keyed by (device name, n, precision, synthesis route) and kept in a
JSON file (``$CNPC_TUNE_CACHE``, default ``~/.cache/cosmonpc_b200/plans.json``)
so a later process reuses them; ``AUTOTUNE = False`` falls back to the fixed
default batch of 8.
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np

AUTOTUNE = True
DEFAULT_BATCH = 8
CANDIDATES = (2, 4, 8, 12, 16, 24)
_lock = threading.Lock()
_plans = None


def cache_path():
    return os.environ.get("CNPC_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "cosmonpc_b200",
                                                         "plans.json"))


def _load():
    global _plans
    if _plans is None:
        try:
            with open(cache_path()) as f:
                _plans = json.load(f)
        except Exception:
            _plans = {}
    return _plans


def _save():
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp%d" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(_plans, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: the plan stays in memory for this process


def _key(n, precision, fused):
    import torch

    return "%s|n%d|%s|%s" % (torch.cuda.get_device_name(), int(n), precision, "fused" if fused else "cufft")


def plans():
    """All cached plans ({key: plan dict})."""
    with _lock:
        return dict(_load())


def fft_batch(n, boxsize, edges, precision):
    """Shell items per synthesis call for this shape class (tuned once)."""
    from . import engine

    if not AUTOTUNE:
        return DEFAULT_BATCH
    fused = engine.fused_shells_apply(n, boxsize, edges, range(len(edges) - 1), precision)
    key = _key(n, precision, fused)
    with _lock:
        p = _load().get(key)
        if p is not None:
            return int(p["fft_batch"])
    import torch

    if torch.cuda.is_current_stream_capturing():
        return DEFAULT_BATCH  # no timing inside a graph capture
    plan = _measure(n, boxsize, edges, precision, fused)
    with _lock:
        _load()[key] = plan
        _save()
    return int(plan["fft_batch"])


def _measure(n, boxsize, edges, precision, fused):
    """Time shell synthesis of 2 x max(candidates) fields at each batch depth."""
    import torch

    from . import _lib, engine

    code, rdt, cdt = engine.PRECISION[precision]
    dev = torch.device("cuda", torch.cuda.current_device())
    # the candidates run on a context of their own, destroyed afterwards: the
    # cuFFT plans of deep batches hold workspaces of several GB each (512^3)
    ctx = _lib.Context(dev.index)
    try:
        with _lib.Context.scope(ctx):
            return _measure_in(ctx, n, boxsize, edges, precision, fused, code, rdt, cdt, dev)
    finally:
        torch.cuda.synchronize()
        ctx.close()
        torch.cuda.empty_cache()


def _measure_in(ctx, n, boxsize, edges, precision, fused, code, rdt, cdt, dev):
    import torch

    from . import _lib, engine

    esz = 4 if precision == "f32" else 8
    per_field = n ** 3 * esz
    per_batch_item = (n * (n // 2) * (n // 4) * 8) if fused else (n * n * (n // 2 + 1) * 2 * esz)
    free = engine.free_device_bytes()
    budget = int(free * 0.5)
    # a call's batch (its spectra or work arrays, and a cuFFT workspace of about
    # the same size) must fit beside the shell fields, which a data vector plans
    # at 80 % of the free memory: at most 10 % of the device per batch
    cap = 0.10 * torch.cuda.get_device_properties(dev).total_memory
    cands = [b for b in CANDIDATES if b * (per_field + per_batch_item) <= budget and 2 * b * per_batch_item <= cap]
    if not cands:
        return {"fft_batch": 1, "ms_per_field": None, "timed": {}}
    nitems = 2 * max(cands)
    while nitems > 1 and nitems * per_field + max(cands) * per_batch_item > budget:
        nitems -= 1
    g = torch.Generator(device=dev).manual_seed(20261203)
    real = torch.randn((n, n, n), generator=g, device=dev, dtype=rdt)
    spec = torch.empty((n, n, n // 2 + 1), dtype=cdt, device=dev)
    ctx.r2c(code, n, 1, real, spec)
    del real
    nb = len(edges) - 1
    keys = [((0, 0, 0, False), b % nb, 0) if i % 2 == 0 else ((2, 0, 0, False), b % nb, 0)
            for i, b in enumerate(range(nitems))]
    timed = {}
    for b in cands:
        sf = None
        try:
            sf = engine.ShellFields(n, boxsize, edges, precision, spec, None, capacity=nitems, fft_batch=b)
            best = None
            for rep in range(4):
                sf.release_all()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                sf.ensure(keys)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                if rep > 0:  # the first repetition makes plans and workspaces
                    best = ms if best is None else min(best, ms)
            timed[str(b)] = best / nitems
        except (_lib.CnpcError, MemoryError, torch.cuda.OutOfMemoryError):
            # a depth whose cuFFT plan or workspace cannot be made is not a candidate
            torch.cuda.synchronize()
        del sf
    torch.cuda.empty_cache()
    if not timed:
        return {"fft_batch": 1, "ms_per_field": None, "timed": {}}
    # the deepest batch within 2 % of the fastest: depths that time alike are
    # run-to-run noise apart, and a deeper batch makes fewer launches
    fastest = min(timed.values())
    win = max((b for b in timed if timed[b] <= 1.02 * fastest), key=int)
    return {"fft_batch": int(win), "ms_per_field": timed[win], "timed": timed}


def block_plan(bins_needed, k_bins, capacity_fields):
    """The block size _plan_blocks chose and why (for reports)."""
    return {"block_size": int(bins_needed), "k_bins": int(k_bins), "fields_resident": int(capacity_fields)}
