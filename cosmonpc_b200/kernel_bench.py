"""Time one library entry point on synthetic device-resident inputs.

    python -m cosmonpc_b200.kernel_bench shells --n 256 --items 8 [--reps 5]
    python -m cosmonpc_b200.kernel_bench gram --n 256 --rows 40 --cols 20 [--tc]
    python -m cosmonpc_b200.kernel_bench paint --n 256 --particles 4000000 --window 4
    python -m cosmonpc_b200.kernel_bench spectral --n 256

Each prints one line: the call, its mean device time (CUDA events over
--reps calls after one warm-up call) and its algorithmic bytes per call.
The inputs are small enough (a few GB at most) to run the same command under
a profiler.
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import _lib, angular, build


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def shells(n, items, reps, boxsize=None, source=0):
    """cnpc_shell_fields: `items` FP32 shell fields (l = 0 and l = 2, 20 bins
    up to k_Nyquist / 2) of one source spectrum (source 0) or of the unit
    spectrum (source 2, the FFT S3 shells)."""
    ctx = _lib.Context.get()
    L = boxsize or 2000.0 * n / 256
    kf = 2 * np.pi / L
    edges = np.linspace(kf, (n / 4 - 0.5) * kf, 21)
    g = torch.Generator(device="cuda").manual_seed(0)
    real = torch.randn((n, n, n), device="cuda", generator=g)
    spec = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    ctx.r2c(_lib.F32, n, 1, real, spec)
    del real
    harms = [angular.harmonic(0, 0), angular.harmonic(2, 0)]
    its = [_lib.ShellItem(j % 20, (j // 20) % 2, 0, source, 1 if source == 2 else 0) for j in range(items)]
    out = torch.empty((items, n, n, n), dtype=torch.float32, device="cuda")
    ms = _time(lambda: ctx.shell_fields(n, L, spec, None, edges, harms, its, [out[j] for j in range(items)]), reps)
    band = n * (n // 2) * (n // 4) * 8
    return {"call": "shell_fields", "n": n, "items": items, "ms": ms, "bytes": items * n ** 3 * 4 + band // 2}


def gram(n, rows, cols, reps, tc=False):
    """cnpc_contract_gram (FP32, CUDA cores) or cnpc_contract_gram_tc (tensor
    cores): rows x cols outputs, the columns a run of the rows."""
    ctx = _lib.Context.get()
    ncell = n ** 3
    g = torch.Generator(device="cuda").manual_seed(1)
    f = torch.randn((max(rows, cols), ncell), device="cuda", generator=g)
    w = torch.randn(ncell, device="cuda", generator=g)
    out = torch.empty((rows, cols), dtype=torch.float64, device="cuda")
    a, b = list(range(rows)), list(range(cols))
    if tc:
        ms = _time(lambda: ctx.gram_tc(ncell, w, f, ncell, a, b, out), reps)
    else:
        ms = _time(lambda: ctx.gram(_lib.F32, ncell, w, f, ncell, a, b, out), reps)
    return {"call": "contract_gram_tc" if tc else "contract_gram", "n": n, "rows": rows, "cols": cols, "ms": ms,
            "bytes": (max(rows, cols) + 1) * ncell * 4}


def paint(n, particles, window, reps):
    """cnpc_paint (FP32, interlaced): a clustered synthetic catalog."""
    from .mocks import lognormal_box

    ctx = _lib.Context.get()
    L = 2000.0 * n / 256
    pos = torch.from_numpy(lognormal_box(particles, L, 20261203)).cuda()
    mesh = torch.empty((2, n, n, n), dtype=torch.float32, device="cuda")
    ms = _time(lambda: ctx.paint(_lib.F32, pos, None, n, L, window, mesh[0], mesh[1]), reps)
    return {"call": "paint", "n": n, "particles": particles, "window": window, "ms": ms,
            "bytes": particles * 24 + 2 * n ** 3 * 4}


def spectral(n, reps):
    """The per-mode spectral passes of a bk_sugi data vector at the 256^3
    workload's binning scaled to n (L = 2000 n / 256, 20 bins 0.01-0.2, k3 bins
    0.02-0.39): cnpc_kbin_counts (k and k3 bins), cnpc_sn_bins_multi (two
    configurations, one S3 source, band 0.4), cnpc_forward_finish (interlaced,
    PCS compensation) and cnpc_field_parity_fold (FP32)."""
    ctx = _lib.Context.get()
    L = 2000.0 * n / 256
    k_edge = np.linspace(0.01, 0.2, 21)
    k3_edge = np.linspace(0.02, 0.4, 41)[:-1]
    g = torch.Generator(device="cuda").manual_seed(2)
    real = torch.randn((n, n, n), device="cuda", generator=g)
    spec = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    spec2 = torch.empty_like(spec)
    ctx.r2c(_lib.F32, n, 1, real, spec)
    ctx.r2c(_lib.F32, n, 1, real, spec2)
    src = torch.empty_like(spec)
    sums = [torch.empty(2 * 41, dtype=torch.float64, device="cuda") for _ in range(2)]
    counts = torch.empty(40, dtype=torch.float64, device="cuda")
    ksum = torch.empty_like(counts)
    half = torch.empty((n // 2 + 1) * n * n, device="cuda")
    nh = n * n * (n // 2 + 1)
    out = {}
    out["kbin_counts_k"] = _time(lambda: ctx.kbin_counts(n, L, k_edge, counts[:20], ksum[:20]), reps)
    out["kbin_counts_k3"] = _time(lambda: ctx.kbin_counts(n, L, k3_edge, counts[:39], ksum[:39]), reps)
    out["sn_bins_multi"] = _time(lambda: ctx.sn_bins_multi(_lib.F32, n, L, spec, spec, 6.4e19, 4, [1e-3, 1e-3],
                                                           [None, angular.harmonic(2, 0, True)], k3_edge, sums,
                                                           [src, None], band=0.4), reps)
    out["forward_finish"] = _time(lambda: ctx.forward_finish(_lib.F32, n, L, spec, spec2, 1.0, _lib.COMP_SINC, 4,
                                                             0.0, 0.0), reps)
    out["parity_fold"] = _time(lambda: ctx.field_parity_fold(_lib.F32, n, real.view(-1), -1, half), reps)
    return {"call": "spectral", "n": n, "ms": out, "bytes": {"sn_bins_multi": 2 * nh * 8, "forward_finish": 3 * nh * 8,
                                                             "parity_fold": (3 * (n // 2) + 1) * n * n * 4}}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["shells", "gram", "paint", "spectral"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--items", type=int, default=8)
    ap.add_argument("--rows", type=int, default=40)
    ap.add_argument("--cols", type=int, default=20)
    ap.add_argument("--particles", type=int, default=4_000_000)
    ap.add_argument("--window", type=int, default=4)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--tc", action="store_true", help="gram: the tensor-core kernel")
    ap.add_argument("--source", type=int, default=0, choices=[0, 2], help="shells: 0 data spectrum, 2 unit spectrum")
    args = ap.parse_args(argv)
    build.build()
    if args.what == "shells":
        r = shells(args.n, args.items, args.reps, source=args.source)
    elif args.what == "gram":
        r = gram(args.n, args.rows, args.cols, args.reps, args.tc)
    elif args.what == "paint":
        r = paint(args.n, args.particles, args.window, args.reps)
    else:
        r = spectral(args.n, args.reps)
    if args.what == "spectral":
        r["GB_per_s"] = {k: b / (r["ms"][k] * 1e6) for k, b in r["bytes"].items()}
    else:
        r["GB_per_s"] = r["bytes"] / (r["ms"] * 1e6)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
