"""Failure detection and the reference's validation errors.

Host-side (no GPU): the run_stats configs the reference rejects raise the same
exception types before any device work (task_executor.py:35-40, :176-196,
param_helper.py:37-59, :90-136), a block plan that cannot fit the device
memory budget raises MemoryError, and library status codes map to Python
exceptions.

Device-side (``gpu``): the FP64 contraction's bounded mbarrier waits are given
a limit of zero polls, so every wait gives up at once; the kernel drains its
own copies, writes NaN, sets the context's status word, and the next call on
the same context (with the normal limit) is correct again.  Nothing waits
without a bound and nothing faults.
"""
import copy

import numpy as np
import pytest


def _box_cfg(tmp_path, **over):
    cfg = dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa", geometry="box-like",
               catalogs={"data_a": str(tmp_path / "none.npy"), "randoms_a": None, "data_b": None,
                         "randoms_b": None},
               column_names=["x", "y", "z"], rsd=[0, 0, 1], apply_rsd=False, nmesh=[64] * 3,
               boxsize=[1000.0] * 3, sampler="tsc", interlaced=True, k_min=0.01, k_max=0.08, k_bins=7,
               angu_config=[0, 0, 0], data_vector_mode="diagonal", shotnoise_mode="ana",
               cosmology={"h": 0.7, "Omega0": 0.3}, redshift_box=0.0, output_dir=str(tmp_path / "out"))
    cfg.update(over)
    return cfg


@pytest.mark.parametrize("over,exc,match", [
    # pk: k_max at or above the Nyquist frequency pi * 64 / 1000 (task_executor.py:35-40)
    (dict(statistic="pk", poles=[0, 2], k_max=0.2011), ValueError, "Nyquist frequency"),
    # bk: 2 k_max at or above the Nyquist frequency (task_executor.py:192-196)
    (dict(k_max=0.101), ValueError, "2 \\* k_max"),
    # ell1 < ell2 (param_helper.py:46-49)
    (dict(angu_config=[0, 2, 2]), ValueError, "ell1 must be greater"),
    # odd ell1 + ell2 + L, odd L, triangle (param_helper.py:50-55)
    (dict(angu_config=[2, 1, 1]), ValueError, "must be even"),
    (dict(angu_config=[1, 1, 1]), ValueError, "must be even"),
    (dict(angu_config=[4, 0, 2]), ValueError, "triangle"),
    # sampler, shot-noise mode, data-vector mode (param_helper.py:104-113, task_executor.py:176-181)
    (dict(sampler="quadratic"), AssertionError, "sampler"),
    (dict(shotnoise_mode="exact"), ValueError, "shotnoise_mode"),
    (dict(data_vector_mode="upper"), ValueError, "data_vector_mode"),
    # odd poles only for a periodic box (task_executor.py:59-63)
    (dict(statistic="pk", poles=[1, 3], k_max=0.1), ValueError, "odd"),
    # tracer type of an auto correlation (param_helper.py:4-16)
    (dict(tracer_type="aab"), AssertionError, "tracer_type"),
    # non-cubic mesh, non-boolean switch (param_helper.py:62-87)
    (dict(nmesh=[64, 64, 32]), AssertionError, "equal"),
    (dict(interlaced=1), TypeError, "boolean"),
])
def test_run_stats_rejects_like_the_reference(tmp_path, over, exc, match):
    """Rejected before any device work: no catalog is read (the path does not exist)."""
    import cosmonpc_b200

    with pytest.raises(exc, match=match):
        cosmonpc_b200.run_stats(_box_cfg(tmp_path, **over))


def test_block_plan_refuses_an_allocation_over_the_budget():
    """A full data vector whose smallest block of shell fields does not fit the
    device-memory budget raises MemoryError instead of allocating."""
    from cosmonpc_b200 import clustering_estimator as ce

    specs = [ce._legs_for_signal(2, 0, 0, 0, "auto", "aaa")]
    with pytest.raises(MemoryError):
        ce._plan_blocks(specs, 20, 256, "f32", "full", False, free_bytes=2 * 4 * 256 ** 3)
    bs, cap = ce._plan_blocks(specs, 20, 256, "f32", "full", False, free_bytes=40 * 4 * 256 ** 3)
    assert 1 <= bs < 20 and cap * 4 * 256 ** 3 <= 0.8 * 40 * 4 * 256 ** 3


class _FakeLib:
    def __init__(self, msg):
        self.msg = msg

    def cnpc_ctx_last_error(self, h):
        return self.msg

    def cnpc_status_string(self, st):
        return b"status"


@pytest.mark.parametrize("status,exc", [(1, ValueError), (2, MemoryError), (3, "CnpcError"), (4, "CnpcError")])
def test_status_codes_map_to_exceptions(status, exc):
    """CNPC_EINVAL -> ValueError, CNPC_ENOMEM -> MemoryError, CNPC_ECUDA and
    CNPC_ECUFFT (e.g. a cuFFT plan that cannot be made) -> CnpcError, with the
    library's message; checked on a fake library handle."""
    from cosmonpc_b200 import _lib

    ctx = _lib.Context.__new__(_lib.Context)
    ctx.lib = _FakeLib(b"cufftPlanMany failed with code 5")
    ctx.h = None
    want = _lib.CnpcError if exc == "CnpcError" else exc
    with pytest.raises(want, match="cufftPlanMany failed"):
        ctx._check(status, "cnpc_fft_c2r")
    ctx._check(0, "ok")


@pytest.mark.gpu
def test_timed_out_device_wait_reports_status_and_context_recovers():
    import torch
    from cosmonpc_b200 import _lib

    ctx = _lib.Context(torch.cuda.current_device())
    try:
        ncell, nf = 32 ** 3, 6
        g = torch.randn(ncell, dtype=torch.float64, device="cuda")
        f = torch.randn((nf, ncell), dtype=torch.float64, device="cuda")
        a, b = [0, 1, 2, 3], [2, 3, 4, 5]
        ref = (g * f[a]) @ f[b].T
        out = torch.zeros((4, 4), dtype=torch.float64, device="cuda")
        ctx.set_wait_limit(0)
        ctx.gram(_lib.F64, ncell, g, f, ncell, a, b, out)
        with pytest.raises(_lib.DeviceTimeout):
            ctx.take_status()
        assert torch.isnan(out).all()
        ctx.take_status()  # the word was cleared by the read
        ctx.set_wait_limit(1 << 22)
        for _ in range(2):
            ctx.gram(_lib.F64, ncell, g, f, ncell, a, b, out)
            ctx.take_status()
            assert torch.allclose(out, ref, rtol=1e-12, atol=1e-9)
    finally:
        ctx.close()


@pytest.mark.gpu
def test_tensor_core_gram_timed_out_wait_reports_status():
    """The tcgen05 Gram's waits given a limit of zero polls: every role gives
    up at its first wait (the producer drains the copies it issued, no MMA is
    issued, TMEM is freed), the outputs are NaN, the status word reports the
    timeout, and the next call with the normal limit is correct."""
    import torch
    from cosmonpc_b200 import _lib

    ctx = _lib.Context(torch.cuda.current_device())
    try:
        ncell, na, nb = 64 ** 3, 12, 8
        g = torch.randn(ncell, dtype=torch.float32, device="cuda")
        f = torch.randn((na, ncell), dtype=torch.float32, device="cuda")
        a, b = list(range(na)), list(range(nb))
        out = torch.zeros((na, nb), dtype=torch.float64, device="cuda")
        ctx.set_wait_limit(0)
        ctx.gram_tc(ncell, g, f, ncell, a, b, out)
        with pytest.raises(_lib.DeviceTimeout):
            ctx.take_status()
        assert torch.isnan(out).all()
        ctx.set_wait_limit(1 << 22)
        ctx.gram_tc(ncell, g, f, ncell, a, b, out)
        ctx.take_status()
        fd, gd = f.double(), g.double()
        ref = (gd * fd[a]) @ fd[b].T
        scale = (gd.abs() * fd[a].abs()) @ fd[b].abs().T
        assert ((out - ref).abs() / scale).max().item() < 2e-6
    finally:
        ctx.close()


@pytest.mark.gpu
def test_timed_out_wait_surfaces_from_the_estimator():
    """A full FP64 data vector whose contraction waits time out raises
    DeviceTimeout when its results are read, instead of returning NaN."""
    from cosmonpc_b200 import _lib, api
    from cosmonpc_b200.mocks import lognormal_box

    pos = lognormal_box(20000, 1000.0, 5, grid=32)
    kw = dict(nmesh=32, boxsize=1000.0, sampler="tsc", interlaced=True, k_min=0.005, k_max=0.045, k_bins=4,
              angu_configs=[(0, 0, 0)], data_vector_mode="full", shotnoise_mode="ana", precision="f64")
    ctx = _lib.Context.get()
    ctx.set_wait_limit(0)
    try:
        with pytest.raises(_lib.DeviceTimeout):
            api.bk_sugi_box_vector(pos, None, **kw)
    finally:
        ctx.set_wait_limit(1 << 22)
        try:
            ctx.take_status()
        except _lib.DeviceTimeout:
            pass
    res = api.bk_sugi_box_vector(pos, None, **kw)[0]
    assert np.isfinite(res["B_sugi"]).all()


@pytest.mark.gpu
def test_autotuned_plan_is_cached_and_exact(tmp_path, monkeypatch):
    """The autotuner times shell-synthesis batch depths for a shape class once,
    caches the winner on disk, and the tuned plan gives the same data vector as
    the fixed default batch."""
    import json

    from cosmonpc_b200 import api, autotune
    from cosmonpc_b200.mocks import lognormal_box

    monkeypatch.setenv("CNPC_TUNE_CACHE", str(tmp_path / "plans.json"))
    monkeypatch.setattr(autotune, "_plans", None)
    pos = lognormal_box(150000, 800.0, 41)
    kw = dict(nmesh=64, boxsize=800.0, sampler="tsc", interlaced=True, k_min=0.01, k_max=0.11, k_bins=8,
              angu_configs=[(0, 0, 0), (2, 0, 2)], data_vector_mode="full", shotnoise_mode="both",
              precision="f32")
    tuned = api.bk_sugi_box_vector(pos, None, **kw)
    saved = json.load(open(tmp_path / "plans.json"))
    assert any("|n64|f32|fused" in k for k in saved)
    plan = next(v for k, v in saved.items() if "|n64|f32|fused" in k)
    assert plan["fft_batch"] in autotune.CANDIDATES and plan["timed"]
    monkeypatch.setattr(autotune, "AUTOTUNE", False)
    fixed = api.bk_sugi_box_vector(pos, None, **kw)
    for a, b in zip(tuned, fixed):
        for key in ("B_sugi", "Bk_raw", "Shot_noise"):
            np.testing.assert_allclose(a[key], b[key], rtol=1e-12, atol=0)
