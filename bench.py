#!/usr/bin/env python
"""Benchmark: Sugiyama bispectrum, box, 256^3 full data vector.

Workload (one "step" = one data vector): a seeded lognormal box catalog of
4e6 particles in a 2000 Mpc/h box, PCS interlaced paint on 256^3, 20 k-bins
over 0.01-0.20 h/Mpc, angular configurations (0,0,0) and (2,0,2) full 20x20
((0,2,2) is their transpose), shot noise "both" (analytical and FFT S3).

value  = seconds per data vector of the fast form (FP32 fields, FP64
         accumulation, shared transforms) with the catalog resident in HBM,
         over K data vectors computed back to back (each one's device work is
         enqueued before the previous one's host algebra runs); "serial" is
         the same with one data vector at a time.
e2e    = the same through the public in-memory API with the catalog in pinned
         host memory: H2D of positions and D2H of the results every step.
plain  = the FP64 per-configuration drop-in on the same catalog (reported,
         with the max relative error of the fast form against it).

Multi-GPU (torchrun): each rank measures its own mock (replicas, weak scaling,
no data-path collective); timing is max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

WORKLOAD = dict(n_particles=4_000_000, boxsize=2000.0, nmesh=256, sampler="pcs", interlaced=True,
                k_min=0.01, k_max=0.20, k_bins=20, angu_configs=[(0, 0, 0), (2, 0, 2)],
                data_vector_mode="full", shotnoise_mode="both")
SMALL = dict(WORKLOAD, n_particles=500_000, nmesh=128, boxsize=1000.0, k_max=0.19, k_bins=12)
# batched mocks: 3 shape classes, CIC interlaced, pk [0,2,4] + bk (0,0,0) diagonal, 15 bins 0.01-0.16
MOCK_CLASSES = [(128, 1000.0), (192, 1500.0), (256, 2000.0)]
MOCKS = dict(n_particles=1_500_000, sampler="cic", interlaced=True, k_min=0.01, k_max=0.16, k_bins=15,
             poles=(0, 2, 4), angu_configs=((0, 0, 0),), data_vector_mode="diagonal", shotnoise_mode="ana")
# DRAM traffic / algorithmic bytes per kernel (ncu dram__bytes_read.sum +
# dram__bytes_write.sum): the contraction from every launch of one 128^3 data
# vector (its traffic scales with cells x staged rows, so the ratio carries to
# 256^3); the shell fields from one 8-field call at 256^3 (column + y/z
# kernels; the last fields' writes still sit in L2 when the kernel ends)
TRAFFIC_RATIO = {"gram": 1.008, "shell_fields": 0.90}
METRIC = "bk_sugi 256^3 full-mode s/data-vector"
UNIT = "s/data-vector"


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region.

    The sampler is started before the region (``start`` + ``wait_first``,
    since nvidia-smi takes a while to print its first sample) and every line
    is time-stamped; ``summary`` keeps the samples between ``mark_start`` and
    ``mark_stop``, plus the first one after the stop, so that a region of a
    few tens of ms still has samples taken under load."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []  # (monotonic time, line)
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def wait_first(self, timeout=5.0):
        t_end = time.monotonic() + timeout
        while self.proc is not None and not self.lines and time.monotonic() < t_end:
            time.sleep(0.01)

    def mark_start(self):
        self.t0 = time.monotonic()

    def mark_stop(self):
        self.t1 = time.monotonic()
        # the first sample after the stop belongs to the region's last 50 ms
        t_end = self.t1 + 0.5
        while self.proc is not None and time.monotonic() < t_end and not any(t > self.t1 for t, _ in self.lines):
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def _window(self):
        if self.t0 is None or self.t1 is None:
            return [ln for _, ln in self.lines]
        inside = [ln for t, ln in self.lines if self.t0 <= t <= self.t1]
        after = [ln for t, ln in self.lines if t > self.t1][:1]
        return inside + after

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self._window():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            err = ""
            if self.proc is not None and self.proc.stderr is not None:
                try:
                    err = self.proc.stderr.read()[:200]
                except Exception:
                    pass
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"],
                    "note": ([ln for _, ln in self.lines[:2]], err)}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- CPU baseline
class CpuBaseline:
    """The oracle port (numpy/scipy, all host threads) timed on bounded samples
    of the workload and extrapolated to one data vector by operation counts.

    The reference computes each angular configuration in its own run_stats call
    (an interlaced paint and the forward transforms each), with shell-field and
    triple-sum counts per configuration as in clustering_estimator.py:867-995
    and :1182-1384.  The interlaced paint is timed once (``paint_s``); every
    sample then times one forward transform, two shell fields and three triple
    sums of the full-size mesh."""

    def __init__(self, workload, seed):
        import numpy as np

        from cosmonpc_b200.mocks import lognormal_box
        from oracle import box as obox

        self.W = workload
        n, L = workload["nmesh"], workload["boxsize"]
        pos = lognormal_box(workload["n_particles"], L, seed)
        w = np.ones(len(pos))
        self.np = len(pos)
        t0 = time.perf_counter()
        self.field = obox.paint_field(pos, w, n, L, workload["sampler"], workload["interlaced"])
        self.paint_s = time.perf_counter() - t0
        self.geo = obox.KGeom(n, L)
        B = workload["k_bins"]
        fields, pairs = 0, 0
        per = 2 if workload["shotnoise_mode"] in ("fft", "both") else 1
        for (l1, l2, L_) in workload["angu_configs"]:
            fields += (B if l1 == l2 else 2 * B) * per
            pairs += (B * (B + 1) // 2 if l1 == l2 else B * B) * per
        self.ncfg = len(workload["angu_configs"])
        self.ffts = self.ncfg * 4  # r2c(delta), c2r(G), r2c/c2r of the S3 source, per configuration
        self.fields, self.pairs = fields, pairs
        # one sample covers this fraction of a data vector's work (paint excluded)
        self.units = 1 + 2 + 3

    def sample(self):
        """Seconds per data vector extrapolated from one timed sample."""
        import numpy as np

        from oracle import angular as oang
        from oracle import box as obox
        from oracle.pmesh_lite import _ifftn

        n, W, geo = self.W["nmesh"], self.W, self.geo
        t0 = time.perf_counter()
        c = obox._fwd(self.field)
        t_fft = time.perf_counter() - t0
        edges = np.linspace(W["k_min"], W["k_max"], W["k_bins"] + 1)
        mask = np.logical_and(geo.knorm >= edges[3], geo.knorm < edges[4])
        y = oang.ylm_function(2, 0, True)(*geo.khat)
        t0 = time.perf_counter()
        F1 = _ifftn(c * y * mask) * float(n) ** 3
        F2 = _ifftn(c * mask) * float(n) ** 3
        t_field = (time.perf_counter() - t0) / 2
        G = np.real(_ifftn(c))
        t0 = time.perf_counter()
        for _ in range(3):
            np.sum(G * F1 * F2)
        t_pair = (time.perf_counter() - t0) / 3
        return self.ncfg * self.paint_s + self.ffts * t_fft + self.fields * t_field + self.pairs * t_pair

    def describe(self):
        return (f"oracle port (numpy/scipy, {os.cpu_count()} host threads) at {self.W['nmesh']}^3: one interlaced "
                f"paint of {self.np} particles ({self.paint_s:.1f} s, timed once), then per sample 1 forward FFT + "
                f"2 shell fields + 3 triple sums, extrapolated to {self.ncfg} configs x (paint + "
                f"{self.ffts // self.ncfg} FFTs) + {self.fields} shell fields + {self.pairs} triple sums")

    def data_vector_fraction(self):
        """Share of one data vector's FFT, shell-field and triple-sum work one sample runs."""
        return self.units / float(self.ffts + self.fields + self.pairs)


def cpu_baseline_estimate(workload, seed, samples=1):
    cb = CpuBaseline(workload, seed)
    vals = [cb.sample() for _ in range(samples)]
    return sum(vals) / len(vals), cb.describe(), os.cpu_count()


def config_of(W, world):
    """The ``config`` object of both arms' JSON lines (identical settings)."""
    return {"workload": "bk_sugi box full %d^3, %.0e lognormal particles, %s interlaced, %d bins %.2f-%.2f, "
                        "(000)+(202) [(022) = transpose], shotnoise %s"
                        % (W["nmesh"], W["n_particles"], W["sampler"].upper(), W["k_bins"], W["k_min"], W["k_max"],
                           W["shotnoise_mode"]),
            "l2": "working set > L2 (shell fields %.1f GB)" % ((3 * W["k_bins"]) * W["nmesh"] ** 3 * 4 / 1e9),
            "parallelism": "replicas x%d" % world}


# ------------------------------------------------------- survey workload
SURVEY = dict(n_data=2_000_000, n_randoms=40_000_000, ra=(100.0, 260.0), dec=(0.0, 60.0), z_mu=0.5,
              z_sigma=0.1, z_clip=(0.2, 0.8), nmesh=512, boxsize=3500.0, sampler="tsc", interlaced=True)


def _survey_runs(seed, reps, scale=1.0):
    """Seconds per run_stats call of the survey cross workload (pk cross [0,2,4];
    bk_sugi aab (0,0,0) and (2,0,2) diagonal), FITS catalogs on local disk,
    FP32 form and the plain FP64 drop-in; each call reads and decodes its
    catalogs like the reference's.  ``scale`` shrinks the catalogs."""
    import tempfile

    import cosmonpc_b200
    from cosmonpc_b200 import mocks

    S = SURVEY
    tmp = tempfile.mkdtemp(prefix="cnpc_survey_")
    geo = dict(ra=S["ra"], dec=S["dec"], z_mu=S["z_mu"], z_sigma=S["z_sigma"], z_clip=S["z_clip"])
    nd, nr = int(S["n_data"] * scale), int(S["n_randoms"] * scale)
    d_a, r_a = mocks.survey_catalogs(nd, nr, seed, **geo)
    d_b, _ = mocks.survey_catalogs(nd // 2, 1000, seed + 1, **geo)  # independent overdensity
    paths = {}
    for key, cols in (("data_a", d_a), ("randoms_a", r_a), ("data_b", d_b)):
        paths[key] = mocks.write_fits_catalog(os.path.join(tmp, key + ".fits"), cols)
    paths["randoms_b"] = paths["randoms_a"]
    base = dict(geometry="survey-like", catalogs=paths, column_names=["RA", "DEC", "Z", "WEIGHT_FKP", "NZ"],
                cosmology={"h": 0.676, "Omega0": 0.31}, compensation=True, nmesh=[S["nmesh"]] * 3,
                boxsize=[S["boxsize"]] * 3, z_range=list(S["z_clip"]), sampler=S["sampler"],
                interlaced=S["interlaced"], comp_weight_plan={"scheme": None, "name_alias": None},
                alpha_scheme="pypower", normalization_scheme="mixed-mesh", output_dir=os.path.join(tmp, "out"))
    runs = {"pk_cross_024": dict(statistic="pk", correlation_mode="cross", k_min=0.005, k_max=0.305, k_bins=30,
                                 poles=[0, 2, 4]),
            "bk_aab_000_diag": dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="aab", k_min=0.01,
                                    k_max=0.21, k_bins=20, angu_config=[0, 0, 0], data_vector_mode="diagonal",
                                    shotnoise_mode="ana"),
            "bk_aab_202_diag": dict(statistic="bk_sugi", correlation_mode="cross", tracer_type="aab", k_min=0.01,
                                    k_max=0.21, k_bins=20, angu_config=[2, 0, 2], data_vector_mode="diagonal",
                                    shotnoise_mode="ana")}
    out = {}
    for name, over in runs.items():
        for prec in ("f32", "f64"):
            cfg = dict(base, **over, precision=prec)
            cosmonpc_b200.run_stats(dict(cfg))  # warm-up: plans, buffers, page cache
            t0 = time.perf_counter()
            for _ in range(reps):
                cosmonpc_b200.run_stats(dict(cfg))
            out["%s:%s" % (name, prec)] = (time.perf_counter() - t0) / reps
    import shutil

    shutil.rmtree(tmp, ignore_errors=True)
    return out, nd, nr


# ----------------------------------------------------------------- main
def _mocks_throughput(per_class, seed, barrier, max_over_ranks, world=1):
    """mocks/s of the fast form (FP32 fields, one paint per mock, the next mock
    queued before the previous one's results are read, each class's device work
    replayed from CUDA graphs captured at the class's largest count) on
    lognormal mocks of Poisson-varying particle counts (mean 1.5e6) resident in
    HBM, and of the plain FP64 per-call path (separate pk and bk calls) on one
    mock per class.  With N ranks each rank runs its own per_class mocks per
    class and the rate is the whole job's (N x mocks over the slowest rank)."""
    import torch

    from cosmonpc_b200 import api, replicas
    from cosmonpc_b200.mocks import lognormal_box

    M = MOCKS
    fast_s, plain_s, total = 0.0, 0.0, 0
    classes = {}
    counts_all = []
    for ci, (n, L) in enumerate(MOCK_CLASSES):
        # mock i of the workload uses seed + i (i = 0..95 over the three classes)
        cats = [torch.from_numpy(lognormal_box(M["n_particles"], L, seed + per_class * ci + i)).cuda()
                for i in range(per_class)]
        counts = [int(c.shape[0]) for c in cats]
        counts_all += counts
        kw = dict(nmesh=n, boxsize=L, sampler=M["sampler"], interlaced=M["interlaced"], k_min=M["k_min"],
                  k_max=M["k_max"], k_bins=M["k_bins"], poles=M["poles"], angu_configs=M["angu_configs"],
                  data_vector_mode=M["data_vector_mode"], shotnoise_mode=M["shotnoise_mode"])
        api.mock_pk_bk(cats[0], None, precision="f32", **kw)  # warm-up: plans and buffers of this class
        graphs = None
        try:  # the device work of a mock replayed from CUDA graphs (captured outside the timed region)
            graphs = api.MockGraphs(max(counts), **kw)
            submit = graphs.submit
            mode = "cuda_graph"
        except RuntimeError:
            submit = lambda c: api.mock_pk_bk(c, None, precision="f32", deferred=True, **kw)
            mode = "eager"
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pending = None
        for c in cats:
            # queue this mock's device work, then read the previous mock's results
            fin = submit(c)
            if pending is not None:
                pending()
            pending = fin
        pending()
        e1.record()
        barrier()
        tf = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
        api.mock_pk_bk_plain(cats[0], None, **kw)
        barrier()
        e0.record()
        api.mock_pk_bk_plain(cats[0], None, **kw)
        e1.record()
        barrier()
        tp = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
        classes["%d^3/L%d" % (n, L)] = {"fast_s_per_mock": tf / len(cats), "plain_s_per_mock": tp, "mode": mode,
                                        "counts": [min(counts), max(counts)]}
        if graphs is not None:
            graphs.close()
        del graphs, submit
        fast_s += tf
        plain_s += tp * len(cats)
        total += len(cats)
        del cats
    return {"value": replicas.job_rate(total, fast_s, world), "unit": "mocks/s",
            "plain_value": replicas.job_rate(total, plain_s, world),
            "speedup": plain_s / fast_s, "mocks": total, "per_class": classes,
            "counts": {"min": min(counts_all), "max": max(counts_all), "mean": sum(counts_all) / len(counts_all)},
            "workload": "pk [0,2,4] + bk_sugi (0,0,0) diagonal, 15 bins 0.01-0.16, CIC interlaced, lognormal "
                        "mocks of Poisson-varying counts (mean 1.5e6); classes 128^3/L1000, 192^3/L1500, "
                        "256^3/L2000"}


def _tuned_plans():
    """Shell-synthesis batch depth per shape class chosen by the autotuner."""
    from cosmonpc_b200 import autotune

    return {k: {"fft_batch": v["fft_batch"], "ms_per_field": v["ms_per_field"]} for k, v in autotune.plans().items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="128^3 profiling case (for ncu captures)")
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mocks", type=int, default=32, help="mocks per shape class for the mocks/s line (0: skip)")
    ap.add_argument("--streams", type=int, default=2, help="CUDA streams the back-to-back data vectors rotate over")
    ap.add_argument("--survey", action="store_true",
                    help="time the survey cross workload (512^3, 2e6 data, 4e7 randoms) instead; one JSON line")
    ap.add_argument("--survey-scale", type=float, default=1.0, help="catalog size factor of --survey")
    ap.add_argument("--survey-steps", type=int, default=1,
                    help="timed run_stats rounds of the survey workload in the default line (0: skip)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    workload = SMALL if args.small else WORKLOAD
    from cosmonpc_b200.mocks import BASE_SEED

    seed = BASE_SEED + 3

    if args.survey:
        import torch

        from cosmonpc_b200.mocks import BASE_SEED as _BS

        t, nd, nr = _survey_runs(_BS + 4, max(1, args.steps), args.survey_scale)
        f32 = sum(v for k, v in t.items() if k.endswith("f32"))
        f64 = sum(v for k, v in t.items() if k.endswith("f64"))
        print(json.dumps({"metric": "survey cross pk + bk aab 512^3 s/data-vector (run_stats, FITS read included)",
                          "value": f32, "unit": "s/data-vector", "higher_is_better": False, "n_gpus": 1,
                          "steps": max(1, args.steps), "plain_f64": f64, "speedup": f64 / f32,
                          "per_call_s": t, "data": "synthetic", "catalogs": {"data": nd, "randoms": nr},
                          "gpu": torch.cuda.get_device_name(0)}))
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        cb = CpuBaseline(workload, seed)
        vals = []
        for i in range(args.warmup + args.steps):
            v = cb.sample()
            if i >= args.warmup:
                vals.append(v)
        value = sum(vals) / len(vals)
        frac = cb.data_vector_fraction()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_of(workload, args.gpus),
                "step_note": "each step is one bounded sample (%.4f of a data vector's transform and triple-sum "
                             "work) extrapolated to a whole data vector; %.3f data vectors' worth of that work "
                             "was timed in all" % (frac, frac * args.steps),
                "data_vectors_timed": frac * args.steps,
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                 "sample": cb.describe()},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    from cosmonpc_b200 import _lib, api, build, replicas
    from cosmonpc_b200.mocks import lognormal_box

    build.build()
    W = workload
    pos_host = lognormal_box(W["n_particles"], W["boxsize"], seed + 1000 * rank)
    pos_pinned = torch.from_numpy(pos_host).pin_memory()
    pos_dev = pos_pinned.cuda()
    common = dict(nmesh=W["nmesh"], boxsize=W["boxsize"], sampler=W["sampler"], interlaced=W["interlaced"],
                  k_min=W["k_min"], k_max=W["k_max"], k_bins=W["k_bins"], angu_configs=W["angu_configs"],
                  data_vector_mode=W["data_vector_mode"], shotnoise_mode=W["shotnoise_mode"])

    def step_resident():
        return api.bk_sugi_box_vector(pos_dev, None, precision="f32", **common)

    sides = [torch.cuda.Stream() for _ in range(max(0, args.streams - 1))]

    def run_vectors(k, pos):
        """k data vectors back to back: each one's device work is enqueued
        before the previous one's host algebra runs (the deferred API), the
        vectors rotating over --streams CUDA streams (each with its own library
        context) so that their kernels can overlap; the current stream waits
        for all of them."""
        cur = torch.cuda.current_stream()
        ring = [cur] + sides
        for s in sides:
            s.wait_stream(cur)
        pending = []
        out = None
        for i in range(k):
            with torch.cuda.stream(ring[i % len(ring)]):
                pending.append(api.bk_sugi_box_vector(pos, None, precision="f32", deferred=True, **common))
            if len(pending) >= max(2, len(ring)):  # one stream: still one vector queued ahead
                out = pending.pop(0)()
        while pending:
            out = pending.pop(0)()
        for s in sides:
            cur.wait_stream(s)
        return out

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x)

    # warm-up in the timed form (two data vectors in flight), so that no
    # allocation of the pipelined run falls inside the timed region
    clk = ClockSampler(local).start()
    run_vectors(args.warmup, pos_dev)
    clk.wait_first()
    barrier()
    # ---- timed region (device resident inputs)
    launches0 = _lib.launch_count
    try:
        barrier()
        clk.mark_start()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        res_fast = run_vectors(args.steps, pos_dev)
        ev1.record()
        barrier()
        clk.mark_stop()
    finally:
        clk.stop()
    t_fast = ev0.elapsed_time(ev1) / 1000.0
    launches = (_lib.launch_count - launches0) // args.steps
    t_fast = max_over_ranks(t_fast)
    # the same data vectors one at a time (host algebra not overlapped)
    barrier()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(args.steps):
        step_resident()
    s1.record()
    barrier()
    t_serial = max_over_ranks(s0.elapsed_time(s1) / 1000.0) / args.steps
    # ---- per-kernel breakdown: a separate pass with every library call
    #      bracketed by CUDA events on the launching stream
    kpass = max(1, min(args.steps, 5))
    _lib.timer = _lib.KernelTimer()
    for _ in range(kpass):
        step_resident()
    torch.cuda.synchronize()
    ksum = _lib.timer.summary()
    _lib.timer = None
    value = t_fast / (args.steps * world)

    # ---- cross-mock amortisation (opt-in): the data-independent unit-spectrum
    #      S3 shells kept across the data vectors of this shape class
    from cosmonpc_b200 import engine as _engine

    _engine.UNIT_SHELL_CACHE = True
    try:
        run_vectors(args.warmup, pos_dev)
        barrier()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        res_amort = run_vectors(args.steps, pos_dev)
        a1.record()
        barrier()
        t_amort = max_over_ranks(a0.elapsed_time(a1) / 1000.0) / (args.steps * world)
    finally:
        _engine.UNIT_SHELL_CACHE = False
        _engine.clear_unit_shell_cache()
    amort_err = 0.0
    for a, b in zip(res_amort, res_fast):
        for k in ("B_sugi", "Bk_raw", "Shot_noise"):
            amort_err = max(amort_err, float(np.max(np.abs(np.asarray(a[k]) - np.asarray(b[k])))
                                             / np.max(np.abs(np.asarray(b[k])))))
    amortized = {"value": t_amort, "unit": UNIT, "max_rel_err_vs_value_path": amort_err,
                 "note": "the FFT S3 unit-spectrum shells (data-independent: nmesh, boxsize, bins, lm) "
                         "synthesised once and kept across data vectors of one shape class"}

    # ---- end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        run_vectors(args.warmup, pos_pinned.numpy())  # warm-up of the host-input path (copy stream, pools)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        r = run_vectors(args.steps, pos_pinned.numpy())
        e1.record()
        barrier()
        t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
        d2h = sum(sum(np.asarray(v).nbytes for k, v in d.items() if k != "SN_terms")
                  + sum(np.asarray(v).nbytes for v in d["SN_terms"].values()) for d in r)
        e2e = {"value": t_e2e / (args.steps * world), "unit": UNIT,
               "h2d_bytes_per_step": int(pos_host.nbytes), "d2h_bytes_per_step": int(d2h)}

    # ---- plain FP64 per-configuration path, and the error of the fast form against it
    plain = None
    max_rel = None
    rel_by_key = None
    if args.plain_steps > 0:
        api.bk_sugi_box_plain(pos_dev, None, **common)  # warm-up: FP64 plans and buffers
        barrier()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record()
        for _ in range(args.plain_steps):
            res_plain = api.bk_sugi_box_plain(pos_dev, None, **common)
        p1.record()
        barrier()
        plain = max_over_ranks(p0.elapsed_time(p1) / 1000.0) / args.plain_steps
        max_rel = 0.0
        rel_by_key = {}
        for cfg, a, b in zip(W["angu_configs"], res_fast, res_plain):
            tag = "%d%d%d" % tuple(cfg)
            pairs = [(k, a[k], b[k]) for k in ("B_sugi", "Bk_raw", "Shot_noise")]
            pairs += [("SN_terms." + k, a["SN_terms"][k], v) for k, v in b["SN_terms"].items()]
            for key, va, vb in pairs:
                den = np.max(np.abs(vb))
                if den > 0:
                    e = float(np.max(np.abs(np.asarray(va) - np.asarray(vb))) / den)
                    rel_by_key[tag + ":" + key] = e
                    max_rel = max(max_rel, e)

    # ---- batched mocks (pk + bk diagonal per mock, three shape classes)
    mocks = None
    if args.mocks > 0:
        mocks = _mocks_throughput(args.mocks, BASE_SEED + 5 + 1000 * rank, barrier, max_over_ranks, world)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return 0

    peak, peak_kind = _peaks()
    ours = {k: v for k, v in ksum.items() if not k.startswith("cufft")}
    dom_name = max(ours, key=lambda k: ours[k][1])
    cnt, tms, nbytes = ksum[dom_name]
    achieved = (nbytes / cnt) / (tms / cnt / 1000.0) / 1e9
    kernels = {k: {"launches_per_step": v[0] // kpass, "ms_per_step": v[1] / kpass,
                   "GB_per_s": (v[2] / (v[1] / 1000.0) / 1e9) if v[1] > 0 and v[2] else None}
               for k, v in sorted(ksum.items(), key=lambda kv: -kv[1][1])}
    cpu = None
    if world == 1 and not args.no_cpu:
        cv, sample, cores = cpu_baseline_estimate(W, seed)
        cpu = {"value": cv, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    survey = None
    if world == 1 and args.survey_steps > 0:
        # the 512^3 FP64 survey path needs most of the device: release this
        # process's pools and contexts and time it in a fresh process
        import gc

        del pos_dev
        _engine.clear_unit_shell_cache()
        _lib.Context.release_all()
        gc.collect()
        torch.cuda.empty_cache()
        proc = subprocess.run([sys.executable, os.path.abspath(__file__), "--survey", "--steps",
                               str(args.survey_steps), "--survey-scale", str(args.survey_scale)],
                              capture_output=True, text=True)
        try:
            sv = json.loads(proc.stdout.strip().splitlines()[-1])
            survey = {"value": sv["value"], "unit": sv["unit"], "plain_f64": sv["plain_f64"],
                      "speedup": sv["speedup"], "catalogs": sv["catalogs"], "per_call_s": sv["per_call_s"],
                      "workload": "survey cross, 512^3, L3500, TSC interlaced, mixed-mesh: pk cross [0,2,4] + "
                                  "bk_sugi aab (000) and (202) diagonal; three run_stats calls, FITS reads "
                                  "included"}
        except Exception:
            survey = {"error": (proc.stderr or proc.stdout)[-400:]}
    mocks_short = None
    if mocks is not None:
        mocks_short = {k: mocks[k] for k in ("value", "unit", "plain_value", "speedup", "mocks")}
    # the summary keys come last, so that a tail of the line still holds them
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_fast / args.steps * 1000.0, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 accumulation", "data": "synthetic",
        "config": config_of(W, world),
        "kernels": kernels,
        "mocks_detail": mocks,
        "plain_rel_err_by_key": rel_by_key,
        "survey": survey,
        "amortized": amortized,
        "plans": _tuned_plans(),
        "serial": {"value": t_serial, "unit": UNIT,
                   "note": "one data vector at a time, host algebra not overlapped with the next vector"},
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (TRAFFIC_RATIO[dom_name] * nbytes / cnt) if dom_name in TRAFFIC_RATIO else None,
                     "traffic_note": "bytes per launch: the kernel's ncu (dram__bytes_read.sum + "
                                     "dram__bytes_write.sum) / algorithmic-bytes ratio times this launch's "
                                     "algorithmic bytes"},
        "e2e": e2e,
        "mocks": mocks_short,
        "plain_f64": {"value": plain, "unit": UNIT, "speedup": (plain / value if plain else None),
                      "max_rel_err_fast_vs_plain": max_rel},
    }
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
