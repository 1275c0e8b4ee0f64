"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference's own golden vectors.

Tolerances: the FP64 path must match to 1e-8 of each multipole's max |value|
(FFT algorithm and summation order are the only differences); the FP32 path
to 1e-5 (the parity bar), or 4x the error single-precision FFTs alone cause on
an ill-conditioned small case where that is larger (conftest.tol); mode
counts bit for bit.
"""
import copy
import glob
import os

import numpy as np
import pytest

from cases import CASES, build_case, flatten_result
from conftest import GOLDEN, parity_report as _report, rel_err, tol

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-8, "f32": 1e-5}


def _run(cfg, precision, tmp_path):
    import cosmonpc_b200

    cfg = copy.deepcopy(cfg)
    cfg["precision"] = precision
    cfg["output_dir"] = str(tmp_path / ("out_" + precision))
    path = cosmonpc_b200.run_stats(cfg)
    return np.load(path, allow_pickle=True).item(), os.path.basename(path)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_golden_case(name, precision, tmp_path):
    cfg, _ = build_case(name, str(tmp_path / "golden"))
    gold = np.load("%s/%s.npz" % (GOLDEN, name))
    res, fname = _run(cfg, precision, tmp_path)
    assert fname == str(gold["output_name"])
    got = flatten_result(res)
    keys = {k for k in gold.files if not k.startswith("checksum") and k != "output_name"}
    assert set(got) == keys
    errs = {}
    for k in sorted(keys):
        if k in ("k_num", "nmodes"):
            np.testing.assert_array_equal(got[k], gold[k])
        else:
            errs[k] = rel_err(got[k], gold[k])
    _report(name, precision, errs)
    bad = {k: e for k, e in errs.items() if not e < tol(precision, name, k)}
    assert not bad, (bad, errs)
    # config keys are carried into the saved dict like the reference does
    assert res["nmesh"] == cfg["nmesh"] and "nyquist_freq" in res


@pytest.mark.parametrize("window", [2, 3, 4])
def test_fp32_tiled_paint_is_bitwise_reproducible(window):
    """The tiled FP32 paint writes each tile's region to a buffer and sums
    every node's contributions in a fixed order, so repeated paints of the
    same catalog give identical meshes; a full data vector then repeats to
    FP64 rounding (its mode sums still add block partials in arrival order)."""
    import torch
    from cosmonpc_b200 import _lib, api
    from cosmonpc_b200.mocks import lognormal_box

    n, L = 64, 640.0
    pos = torch.from_numpy(lognormal_box(300000, L, 17 + window)).cuda()
    ctx = _lib.Context.get()
    meshes = []
    for _ in range(3):
        m = torch.empty((2, n, n, n), dtype=torch.float32, device="cuda")
        ctx.paint(_lib.F32, pos, None, n, L, window, m[0], m[1])
        meshes.append(m)
    assert torch.equal(meshes[0], meshes[1]) and torch.equal(meshes[0], meshes[2])
    if window == 4:
        kw = dict(nmesh=n, boxsize=L, sampler="pcs", interlaced=True, k_min=0.02, k_max=0.14, k_bins=6,
                  angu_configs=[(0, 0, 0), (2, 0, 2)], data_vector_mode="full", shotnoise_mode="both",
                  precision="f32")
        a = api.bk_sugi_box_vector(pos, None, **kw)
        b = api.bk_sugi_box_vector(pos, None, **kw)
        for x, y in zip(a, b):
            for key in ("B_sugi", "Bk_raw", "Shot_noise"):
                np.testing.assert_allclose(x[key], y[key], rtol=1e-12, atol=0, err_msg=key)


@pytest.mark.parametrize("n,npart", [(24, 5000), (40, 20000)])
@pytest.mark.parametrize("window", [1, 2, 3, 4])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_paint_matches_oracle(window, precision, n, npart):
    """Per-particle paint (small n) and the tiled shared-memory paint (FP32,
    n >= 32 with enough particles; n = 40 also has a partial edge tile)."""
    import torch
    from cosmonpc_b200 import _lib, engine
    from oracle.pmesh_lite import paint_mass

    L = 300.0
    rng = np.random.default_rng(window)
    pos = rng.random((npart, 3)) * L
    pos[:7] = [[0, 0, 0], [L * (1 - 1e-16), 1, 2], [L / n * 3, L / n * 5.5, 0.5 * L], [1e-9, 299.9, 150],
               [L / 2, L / 2, L / 2], [L / n * 7.25, 0.0, L / n * 11.75], [L - 1e-7, L - 1e-7, L - 1e-7]]
    w = 0.5 + rng.random(npart)
    ctx = _lib.Context.get()
    code, rdt, _ = engine.PRECISION[precision]
    mesh = torch.empty((2, n, n, n), dtype=rdt, device="cuda")
    ctx.paint(code, torch.from_numpy(pos).cuda(), torch.from_numpy(w).cuda(), n, L, window, mesh[0], mesh[1])
    g = pos * (n / L)
    for k, shift in enumerate((0.0, 0.5)):
        ref = paint_mass(g + shift, w, [n] * 3, window)
        got = mesh[k].double().cpu().numpy()
        tol = 1e-12 if precision == "f64" else 2e-6
        assert np.max(np.abs(got - ref)) < tol * np.max(ref)
        assert abs(got.sum() - ref.sum()) < tol * w.sum() * 10
        # mass is conserved except for the NGP exact-tie particle planted above
        if window > 1:
            assert abs(got.sum() - w.sum()) < tol * w.sum() * 10


@pytest.mark.parametrize("n,L,k_min,k_max,bins", [(64, 1000.0, 0.005, 0.195, 19), (128, 1000.0, 0.01, 0.2, 19),
                                                  (256, 2000.0, 0.01, 0.2, 20), (256, 2000.0, 0.02, 0.4, 19)])
def test_mode_counts_bit_exact(n, L, k_min, k_max, bins):
    from cosmonpc_b200 import engine
    from oracle.box import KGeom, kbin_count

    edges = np.linspace(k_min, k_max, bins + 1)
    c, s = engine.kbin_counts(n, L, edges)
    geo = KGeom(n, L)
    rc, rs = kbin_count(bins, edges, geo.knorm)
    np.testing.assert_array_equal(c.cpu().numpy(), rc)
    np.testing.assert_allclose(s.cpu().numpy(), rs, rtol=1e-12)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_bk_full_64_against_oracle(precision, tmp_path):
    """A larger full-mode case (64^3, 12 bins, PCS interlaced, 3e5 particles)."""
    from cosmonpc_b200.mocks import lognormal_box, write_npy_catalog
    from oracle.driver import run_box

    pos = lognormal_box(300000, 1000.0, 77, grid=64)
    path = write_npy_catalog(str(tmp_path / "cat.npy"), pos)
    cfg = dict(statistic="bk_sugi", correlation_mode="auto", tracer_type="aaa", geometry="box-like",
               catalogs={"data_a": path, "randoms_a": None, "data_b": None, "randoms_b": None},
               column_names=["x", "y", "z"], rsd=[0, 0, 1], apply_rsd=False, nmesh=[64] * 3,
               boxsize=[1000.0] * 3, sampler="pcs", interlaced=True, k_min=0.01, k_max=0.1, k_bins=12,
               angu_config=[2, 0, 2], data_vector_mode="full", shotnoise_mode="both", block_size=5,
               cosmology={"h": 0.7, "Omega0": 0.3}, redshift_box=0.0)
    ref = flatten_result(run_box(copy.deepcopy(cfg)))
    res, _ = _run(cfg, precision, tmp_path)
    got = flatten_result(res)
    for k in ref:
        if k == "nmodes":
            np.testing.assert_array_equal(got[k], ref[k])
        else:
            assert rel_err(got[k], ref[k]) < TOL[precision], (k, rel_err(got[k], ref[k]))


@pytest.mark.parametrize("n", [64, 128, 192, 256])
def test_fused_shell_fields_match_cufft_route(n):
    """cnpc_shell_fields (band-limited fused transform) against shell spectra
    followed by cuFFT C2R, for every harmonic kind, component, source and conj."""
    import torch
    from cosmonpc_b200 import _lib, angular

    L = 1000.0 * n / 64
    kf = 2 * np.pi / L
    edges = np.linspace(0.0, (n / 4 - 0.5) * kf, 6)
    ctx = _lib.Context.get()
    rng = np.random.default_rng(n)
    specs = []
    for _ in range(2):
        real = torch.from_numpy(rng.standard_normal((n, n, n)).astype(np.float32)).cuda()
        sp = torch.empty((n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
        ctx.r2c(_lib.F32, n, 1, real, sp)
        specs.append(sp)
    harms = [angular.harmonic(0, 0), angular.harmonic(2, 1), angular.harmonic(1, 1), angular.harmonic(3, -2),
             angular.harmonic(4, 0)]
    # (harmonic, component) pairs whose field is not identically zero
    comps = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (3, 0), (3, 1), (4, 0)]
    items = []
    for j in range(10):
        hi, c = comps[j % len(comps)]
        items.append(_lib.ShellItem(j % 5, hi, c, j % 3, (j // 3) % 2))
    half = torch.empty((len(items), n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    ctx.shell_spectra(_lib.F32, n, L, specs[0], specs[1], edges, harms, items, half)
    assert half.abs().amax(dim=(1, 2, 3)).min().item() > 0
    ref = torch.empty((len(items), n, n, n), dtype=torch.float32, device="cuda")
    ctx.c2r(_lib.F32, n, len(items), half, ref)
    torch.cuda.synchronize()
    del half
    out = torch.empty_like(ref)
    ctx.shell_fields(n, L, specs[0], specs[1], edges, harms, items, [out[j] for j in range(len(items))])
    torch.cuda.synchronize()
    for j in range(len(items)):
        a, b = out[j].double(), ref[j].double()
        scale = b.abs().max().item()
        assert scale > 0
        assert (a - b).abs().max().item() < 2e-6 * scale, (j, (a - b).abs().max().item() / scale)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("n", [24, 64])
def test_pair_contraction_matches_fp64_sums(dtype, n):
    """cnpc_contract_pairs against FP64 torch sums of G F_a F_b, with repeated
    fields, pairs split over several chunks and a padded field stride."""
    import torch
    from cosmonpc_b200 import _lib

    code, tdt = (_lib.F32, torch.float32) if dtype == "f32" else (_lib.F64, torch.float64)
    ncell, stride, nf = n ** 3, n ** 3 + 8, 7
    g = torch.randn(ncell, dtype=torch.float64, device="cuda")
    f = torch.randn((nf, stride), dtype=torch.float64, device="cuda")
    a = [0, 1, 2, 3, 4, 5, 6, 0, 3, 6, 2, 1, 5]
    b = [0, 1, 2, 3, 4, 5, 6, 1, 4, 0, 2, 6, 3]
    out = torch.empty(len(a), dtype=torch.float64, device="cuda")
    ctx = _lib.Context.get()
    ctx.contract_pairs(code, ncell, g.to(tdt), f.to(tdt), stride, a, b, out)
    gl, fl = g.to(tdt).double(), f.to(tdt).double()
    ref = torch.stack([(gl * fl[i, :ncell] * fl[j, :ncell]).sum() for i, j in zip(a, b)])
    scale = torch.stack([(gl.abs() * fl[i, :ncell].abs() * fl[j, :ncell].abs()).sum() for i, j in zip(a, b)])
    err = ((out - ref).abs() / scale).max().item()
    assert err < (1e-14 if dtype == "f64" else 1e-6), err


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("n,offset", [(30, 0), (64, 0), (128, 0), (256, 0), (192, 0), (64, 1)])
def test_parity_fold_matches_torch(dtype, n, offset):
    """cnpc_field_parity_fold bit for bit against torch: the planes 0 and n/2
    copied, the others in[x] + sign in[n - x][-y][-z]; the row kernel (FP32,
    n % 4 == 0, 16-byte aligned) and the element kernel (odd n / 4, an
    unaligned input, FP64)."""
    import torch
    from cosmonpc_b200 import _lib

    code, tdt = (_lib.F32, torch.float32) if dtype == "f32" else (_lib.F64, torch.float64)
    ctx = _lib.Context.get()
    g = torch.Generator(device="cuda").manual_seed(n + offset)
    buf = torch.randn(n ** 3 + offset, dtype=tdt, device="cuda", generator=g)
    src = buf[offset:]
    x = src.view(n, n, n)
    # index (n - i) mod n along y and z, plane n - x along x
    rev = torch.roll(torch.flip(x, dims=(1, 2)), shifts=(1, 1), dims=(1, 2))
    for sign in (1, -1):
        out = torch.full(((n // 2 + 1) * n * n,), float("nan"), dtype=tdt, device="cuda")
        ctx.field_parity_fold(code, n, src, sign, out)
        ref = x[: n // 2 + 1].clone()
        ref[1: n // 2] = x[1: n // 2] + sign * torch.flip(rev[n // 2 + 1:], dims=(0,))
        torch.cuda.synchronize()
        assert torch.equal(out.view(n // 2 + 1, n, n), ref), (dtype, n, offset, sign)


@pytest.mark.parametrize("n", [64, 128])
def test_parity_folded_contraction_matches_full_sum(n):
    """Shells of the unit spectrum have the parity (-1)^l, so sum_x G F_a F_b
    over all cells equals the sum over the planes x <= n/2 of the folded weight
    (cnpc_field_parity_fold, sign (-1)^(l_a + l_b)); checked for even and odd
    products, with fields from the fused kernel (its reflected planes) and the
    cuFFT route."""
    import torch
    from cosmonpc_b200 import _lib, angular

    L = 1000.0 * n / 64
    kf = 2 * np.pi / L
    edges = np.linspace(0.0, (n / 4 - 0.5) * kf, 5)
    ctx = _lib.Context.get()
    harms = [angular.harmonic(0, 0), angular.harmonic(1, 0), angular.harmonic(2, 0)]
    # unit-spectrum items (source 2, conj): l = 0, 1, 2 over 4 bins
    items = [_lib.ShellItem(b, h, 1 if h == 1 else 0, 2, 1) for h in range(3) for b in range(4)]
    ls = [angular_l for angular_l in (0, 1, 2) for _ in range(4)]
    fused = torch.empty((len(items), n ** 3), dtype=torch.float32, device="cuda")
    ctx.shell_fields(n, L, None, None, edges, harms, items, [fused[j] for j in range(len(items))])
    half = torch.empty((len(items), n, n, n // 2 + 1), dtype=torch.complex64, device="cuda")
    ctx.shell_spectra(_lib.F32, n, L, None, None, edges, harms, items, half)
    direct = torch.empty((len(items), n ** 3), dtype=torch.float32, device="cuda")
    ctx.c2r(_lib.F32, n, len(items), half, direct)
    del half
    rng = np.random.default_rng(n)
    G = torch.from_numpy(rng.standard_normal(n ** 3).astype(np.float32)).cuda()
    hcell = (n // 2 + 1) * n * n
    for fields in (fused, direct):
        for (la, lb) in ((0, 0), (2, 0), (1, 1), (1, 0), (2, 1)):
            a = [j for j in range(len(items)) if ls[j] == la]
            b = [j for j in range(len(items)) if ls[j] == lb]
            full = torch.empty((len(a), len(b)), dtype=torch.float64, device="cuda")
            ctx.gram(_lib.F32, n ** 3, G, fields, n ** 3, a, b, full)
            Gf = torch.empty(hcell, dtype=torch.float32, device="cuda")
            ctx.field_parity_fold(_lib.F32, n, G, -1 if (la + lb) % 2 else 1, Gf)
            folded = torch.empty_like(full)
            ctx.gram(_lib.F32, hcell, Gf, fields, n ** 3, a, b, folded)
            fd, gd = fields.double(), G.double()
            scale = (gd.abs() * fd[a].abs()) @ fd[b].abs().T
            err = ((folded - full).abs() / scale).max().item()
            assert err < 2e-6, (la, lb, err)


@pytest.mark.parametrize("ncell,na,nb,shared", [(128 ** 3, 40, 20, True), (256 ** 3, 40, 20, True),
                                                (64 ** 3 + 100, 17, 9, False), (4096 + 36, 3, 2, False)])
def test_ffma_gram_matches_fp64(ncell, na, nb, shared):
    """cnpc_contract_gram in FP32 (CUDA-core FFMA kernel: FP32 partials over
    512 cells per lane, folded into FP64) against FP64 sums of the same FP32
    inputs, relative to sum |G F_a F_b|; at 256^3 every warp folds many
    times."""
    import torch
    from cosmonpc_b200 import _lib

    rng = np.random.default_rng(ncell + 7 * na + nb)
    nf = na if shared else na + nb
    stride = (ncell + 3) // 4 * 4
    f = torch.from_numpy(rng.standard_normal((nf, stride)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.standard_normal(ncell).astype(np.float32)).cuda()
    a = list(range(na))
    b = list(range(nb)) if shared else list(range(na, na + nb))
    ctx = _lib.Context.get()
    out = torch.empty((na, nb), dtype=torch.float64, device="cuda")
    ctx.gram(_lib.F32, ncell, g, f, stride, a, b, out)
    fd, gd = f[:, :ncell].double(), g.double()
    ref = (gd * fd[a]) @ fd[b].T
    scale = (gd.abs() * fd[a].abs()) @ fd[b].abs().T
    err = ((out - ref).abs() / scale).max().item()
    assert err < 1e-6, err


@pytest.mark.parametrize("ncell,na,nb,shared", [(4096 + 36, 1, 1, False), (32 ** 3, 8, 8, True),
                                                (64 ** 3, 40, 20, True), (64 ** 3, 40, 24, False),
                                                (48 ** 3, 24, 20, False), (64 ** 3 + 100, 17, 9, False),
                                                (128 ** 3, 40, 20, True), (100, 3, 2, False)])
def test_tensor_core_gram_matches_fp64(ncell, na, nb, shared):
    """cnpc_contract_gram_tc (TF32 pairs on tcgen05, A operand in tensor
    memory) against FP64 sums of the same FP32 inputs and against the CUDA-core
    FFMA Gram, with ragged last chunks (and a call smaller than one chunk),
    rows and columns short of the 40 x 24 window, shared row/column fields, a
    padded field stride, and at 128^3 many accumulator periods per block."""
    import torch
    from cosmonpc_b200 import _lib

    rng = np.random.default_rng(ncell + na + nb)
    nf = na if shared else na + nb
    stride = (ncell + 7) // 4 * 4 + 4
    f = torch.from_numpy(rng.standard_normal((nf, stride)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.standard_normal(ncell).astype(np.float32)).cuda()
    a = list(rng.permutation(nf)[:na])
    b = [a[(3 * j) % na] for j in range(nb)] if shared else list(range(na, na + nb))
    ctx = _lib.Context.get()
    out = torch.empty((na, nb), dtype=torch.float64, device="cuda")
    ctx.gram_tc(ncell, g, f, stride, a, b, out)
    fd, gd = f[:, :ncell].double(), g.double()
    ref = (gd * fd[a]) @ fd[b].T
    scale = (gd.abs() * fd[a].abs()) @ fd[b].abs().T
    err = ((out - ref).abs() / scale).max().item()
    assert err < 2e-6, err
    if na + nb <= 40:  # the FFMA kernel's staging limit
        ff = torch.empty_like(out)
        ctx.gram(_lib.F32, ncell, g, f, stride, a, b, ff)
        err_ff = ((ff - ref).abs() / scale).max().item()
        assert err < 4 * err_ff + 1e-7, (err, err_ff)


@pytest.mark.parametrize("case", ["clustered", "heavy_weights", "light_weights", "overfull_cell"])
def test_tiled_paint_fixed_point_scales(case):
    """The tiled FP32 paint's per-tile fixed-point scale against the FP64
    oracle paint: a clustered catalog, weights of 1e3 and of 1e-9 (scale 2^60
    and more), and 150000 particles in one cell (window count above 65536: the
    tile accumulates in FP32, so the check is at the level of FP32 sums of
    1.5e5 deposits)."""
    import torch
    from cosmonpc_b200 import _lib
    from oracle.pmesh_lite import paint_mass

    n, L, window = 64, 640.0, 4
    rng = np.random.default_rng(len(case))
    if case == "clustered":
        centres = rng.random((40, 3)) * L
        pos = (centres[rng.integers(0, 40, 120000)] + rng.normal(0, 6.0, (120000, 3))) % L
        w = 0.5 + rng.random(len(pos))
    elif case == "heavy_weights":
        pos = 100.0 + rng.random((60000, 3)) * 150.0
        w = 1e3 * (0.5 + rng.random(len(pos)))
    elif case == "overfull_cell":
        pos = 205.0 + rng.random((150000, 3)) * 9.0  # inside cell (20, 20, 20)
        w = 0.5 + rng.random(len(pos))
    else:
        pos = rng.random((60000, 3)) * L
        w = 1e-9 * (0.5 + rng.random(len(pos)))
    ctx = _lib.Context.get()
    mesh = torch.empty((2, n, n, n), dtype=torch.float32, device="cuda")
    ctx.paint(_lib.F32, torch.from_numpy(pos).cuda(), torch.from_numpy(w).cuda(), n, L, window, mesh[0], mesh[1])
    g = pos * (n / L)
    for k, shift in enumerate((0.0, 0.5)):
        ref = paint_mass(g + shift, w, [n] * 3, window)
        got = mesh[k].double().cpu().numpy()
        tol = 2e-4 if case == "overfull_cell" else 2e-6
        assert np.max(np.abs(got - ref)) < tol * np.max(ref), (case, k)
        assert abs(got.sum() - w.sum()) < (1e-4 if case == "overfull_cell" else 1e-6) * w.sum()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("aliased", [True, False])
def test_forward_finish_band_copy(dtype, aliased):
    """cnpc_forward_finish_band: the finished spectrum equals cnpc_forward_finish
    bit for bit, and the band copy (written over the twin spectrum, or to a
    separate buffer) is that spectrum zeroed at |k| >= the band, |k| as the
    oracle computes it."""
    import torch
    from cosmonpc_b200 import _lib
    from oracle.box import KGeom

    n, L = 32, 400.0
    code = _lib.F64 if dtype == "f64" else _lib.F32
    cdt = torch.complex128 if dtype == "f64" else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(3)
    shape = (n, n, n // 2 + 1)
    s1 = torch.randn(shape, dtype=cdt, device="cuda", generator=g)
    s2 = torch.randn(shape, dtype=cdt, device="cuda", generator=g)
    ctx = _lib.Context.get()
    ref = s1.clone()
    ctx.forward_finish(code, n, L, ref, s2.clone(), 0.7, _lib.COMP_SINC, 3, 1.25)
    band = 9.5 * 2 * np.pi / L
    a, b = s1.clone(), s2.clone()
    out = b if aliased else torch.empty_like(a)
    ctx.forward_finish_band(code, n, L, a, b, 0.7, _lib.COMP_SINC, 3, 1.25, 0.0, out, band)
    assert torch.equal(torch.view_as_real(a), torch.view_as_real(ref))
    kn = torch.from_numpy(np.ascontiguousarray(KGeom(n, L).knorm[:, :, :n // 2 + 1])).cuda()
    expect = torch.where(kn < band, ref, torch.zeros_like(ref))
    assert torch.equal(torch.view_as_real(out), torch.view_as_real(expect))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("cross", [False, True])
def test_sn_bins_multi_matches_single_calls(dtype, cross):
    """cnpc_sn_bins_multi (two shot-noise configurations in one pass: sn0 with
    Y_00 and a source, sn0 = 0 with Y_20 and a source) against one
    cnpc_sn_bins call per configuration: the same source spectra bit for bit,
    the same shell sums and source totals up to summation order."""
    import torch
    from cosmonpc_b200 import _lib, angular

    n, L = 48, 600.0
    code = _lib.F64 if dtype == "f64" else _lib.F32
    cdt = torch.complex128 if dtype == "f64" else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(7 + cross)
    shape = (n, n, n // 2 + 1)
    a = torch.randn(shape, dtype=cdt, device="cuda", generator=g)
    b = torch.randn(shape, dtype=cdt, device="cuda", generator=g) if cross else a
    kf = 2 * np.pi / L
    edges = np.linspace(2 * kf, 17.5 * kf, 12)
    band = 14.2 * kf
    nb = len(edges) - 1
    ctx = _lib.Context.get()
    cfgs = [(1234.5, None), (0.0, angular.harmonic(2, 0, True))]
    sums_m = [torch.empty(2 * (nb + 1), dtype=torch.float64, device="cuda") for _ in cfgs]
    src_m = [torch.empty(shape, dtype=cdt, device="cuda") for _ in cfgs]
    ctx.sn_bins_multi(code, n, L, a, b, 3.5, 3, [c[0] for c in cfgs], [c[1] for c in cfgs], edges,
                      sums_m, src_m, band=band)
    for (sn0, y), sm, srm in zip(cfgs, sums_m, src_m):
        s1 = torch.empty(2 * (nb + 1), dtype=torch.float64, device="cuda")
        sr1 = torch.empty(shape, dtype=cdt, device="cuda")
        ctx.sn_bins(code, n, L, a, b, 3.5, sn0, 3, y, edges, s1, source=sr1, band=band)
        assert torch.equal(torch.view_as_real(srm), torch.view_as_real(sr1))
        scale = s1[0::2].abs().max().item()
        assert scale > 0
        assert ((sm[0::2] - s1[0::2]).abs().max().item()) <= 1e-12 * scale
    # a configuration without source next to one with a source
    s_ns = torch.empty(2 * nb, dtype=torch.float64, device="cuda")
    s_src = torch.empty(2 * (nb + 1), dtype=torch.float64, device="cuda")
    sr = torch.empty(shape, dtype=cdt, device="cuda")
    ctx.sn_bins_multi(code, n, L, a, b, 3.5, 3, [0.0, 1234.5], [cfgs[1][1], None], edges, [s_ns, s_src],
                      [None, sr], band=band)
    assert torch.equal(torch.view_as_real(sr), torch.view_as_real(src_m[0]))
    scale = sums_m[1][0::2].abs().max().item()
    assert (s_ns[0::2] - sums_m[1][0::2][:nb]).abs().max().item() <= 1e-12 * scale


@pytest.mark.parametrize("ngs,rows,nb,shared", [(2, (20, 20), 20, True), (3, (5, 9, 11), 8, False),
                                                (1, (17,), 7, False), (4, (10, 10, 10, 10), 20, True)])
def test_tensor_core_multi_weight_gram(ngs, rows, nb, shared):
    """cnpc_contract_gram_tc_multi_g (a weight field per row, tensor cores)
    against FP64 sums and against the CUDA-core multi-weight Gram."""
    import torch
    from cosmonpc_b200 import _lib

    n = 64
    ncell = n ** 3
    rng = np.random.default_rng(ngs * 1000 + nb)
    na = sum(rows)
    nf = na + (0 if shared else nb)
    stride = ncell + 4
    f = torch.from_numpy(rng.standard_normal((nf, stride)).astype(np.float32)).cuda()
    gs = [torch.from_numpy(rng.standard_normal(ncell).astype(np.float32)).cuda() for _ in range(ngs)]
    a = list(rng.permutation(na))
    ag = [g for g, r in enumerate(rows) for _ in range(r)]
    b = a[:nb] if shared else list(range(na, na + nb))
    ctx = _lib.Context.get()
    out = torch.empty((na, nb), dtype=torch.float64, device="cuda")
    ctx.gram_tc_multi_g(ncell, gs, f, stride, a, ag, b, out)
    ff = torch.empty_like(out)
    ctx.gram_multi_g(ncell, gs, f, stride, a, ag, b, ff)
    fd = f[:, :ncell].double()
    gw = torch.stack([gs[g].double() for g in ag])
    ref = (gw * fd[a]) @ fd[b].T
    scale = (gw.abs() * fd[a].abs()) @ fd[b].abs().T
    assert ((out - ref).abs() / scale).max().item() < 2e-6
    assert ((out - ff).abs() / scale).max().item() < 2e-6


@pytest.mark.parametrize("ngs,rows,nb,shared", [(2, (20, 20), 20, True), (3, (5, 9, 11), 8, False),
                                                (1, (17,), 7, False), (4, (10, 10, 10, 10), 20, True)])
def test_multi_weight_gram_matches_separate_launches(ngs, rows, nb, shared):
    """cnpc_contract_gram_multi_g (several weight fields, rows weighted per
    group, columns shared) against one cnpc_contract_gram per weight field and
    against FP64 sums."""
    import torch
    from cosmonpc_b200 import _lib

    n = 48
    ncell = n ** 3
    rng = np.random.default_rng(ngs * 100 + nb)
    na = sum(rows)
    nf = na + (0 if shared else nb)
    stride = ncell + 4
    f = torch.from_numpy(rng.standard_normal((nf, stride)).astype(np.float32)).cuda()
    gs = [torch.from_numpy(rng.standard_normal(ncell).astype(np.float32)).cuda() for _ in range(ngs)]
    a = list(rng.permutation(na))
    ag = [g for g, r in enumerate(rows) for _ in range(r)]
    b = a[:nb] if shared else list(range(na, na + nb))
    ctx = _lib.Context.get()
    out = torch.empty((na, nb), dtype=torch.float64, device="cuda")
    ctx.gram_multi_g(ncell, gs, f, stride, a, ag, b, out)
    fd = f[:, :ncell].double()
    r0 = 0
    for g, r in enumerate(rows):
        rr = a[r0:r0 + r]
        sep = torch.empty((r, nb), dtype=torch.float64, device="cuda")
        ctx.gram(_lib.F32, ncell, gs[g], f, stride, rr, b, sep)
        ref = (gs[g].double() * fd[rr]) @ fd[b].T
        scale = (gs[g].double().abs() * fd[rr].abs()) @ fd[b].abs().T
        got = out[r0:r0 + r]
        assert ((got - ref).abs() / scale).max().item() < 1e-6
        assert ((got - sep).abs() / scale).max().item() < 1e-6
        r0 += r


@pytest.mark.parametrize("shotnoise_mode", ["ana", "both"])
def test_mock_graphs_match_eager(shotnoise_mode):
    """MockGraphs (the mock pipeline replayed from CUDA graphs, two slots)
    against eager mock_pk_bk on catalogs of uneven (Poisson-varying) particle
    counts, replayed back to back; a catalog above the capacity is refused, and
    with FFT shot noise of (0,0,0) only the captured count is accepted."""
    import torch
    from cosmonpc_b200 import api
    from cosmonpc_b200.mocks import lognormal_box

    n, L = 64, 500.0
    kw = dict(sampler="cic", interlaced=True, k_min=0.01, k_max=0.16, k_bins=15, poles=(0, 2, 4),
              angu_configs=((0, 0, 0),), data_vector_mode="diagonal", shotnoise_mode=shotnoise_mode)
    cats = [torch.from_numpy(lognormal_box(100000, L, 900 + i)).cuda() for i in range(4)]
    counts = [int(c.shape[0]) for c in cats]
    if shotnoise_mode == "ana":
        assert len(set(counts)) == len(counts)  # Poisson-varying
        graphs = api.MockGraphs(max(counts) + 17, n, L, **kw)
    else:
        cats = [c[:min(counts)] for c in cats]
        graphs = api.MockGraphs(min(counts), n, L, **kw)
    pending, got = None, []
    for c in cats:
        fin = graphs.submit(c)
        if pending is not None:
            got.append(pending())
        pending = fin
    got.append(pending())
    for c, (pk, bks) in zip(cats, got):
        ref_pk, ref_bks = api.mock_pk_bk(c, None, nmesh=n, boxsize=L, **kw)
        for key in ("P0", "P2", "P4"):
            assert rel_err(pk[key], ref_pk[key]) < 1e-6, key
        for bk, ref in zip(bks, ref_bks):
            keys = ("B_sugi", "Bk_raw", "Shot_noise") + (("SN3_FFT",) if shotnoise_mode == "both" else ())
            for key in keys:
                g = bk["SN_terms"][key] if key == "SN3_FFT" else bk[key]
                r = ref["SN_terms"][key] if key == "SN3_FFT" else ref[key]
                assert rel_err(g, r) < 1e-6, key
            assert bk["I_norm"] == pytest.approx(ref["I_norm"], rel=1e-15)
    with pytest.raises(ValueError):
        graphs.submit(torch.cat([cats[0], cats[1]]))
    if shotnoise_mode == "both":
        with pytest.raises(ValueError):
            graphs.submit(cats[0][:-1])
    graphs.close()


def test_unit_shell_cache_matches_fresh_shells():
    """With the opt-in unit-shell cache the FFT S3 shells of a full data vector
    are synthesised once and reused: later calls equal calls without it."""
    from cosmonpc_b200 import api, engine
    from cosmonpc_b200.mocks import lognormal_box

    pos = lognormal_box(200000, 800.0, 31)
    kw = dict(nmesh=64, boxsize=800.0, sampler="tsc", interlaced=True, k_min=0.01, k_max=0.11, k_bins=8,
              angu_configs=[(0, 0, 0), (2, 0, 2)], data_vector_mode="full", shotnoise_mode="both",
              precision="f32")
    ref = api.bk_sugi_box_vector(pos, None, **kw)
    engine.UNIT_SHELL_CACHE = True
    try:
        runs = [api.bk_sugi_box_vector(pos, None, **kw) for _ in range(3)]
        assert engine._unit_shells and engine._unit_origin
    finally:
        engine.UNIT_SHELL_CACHE = False
        engine.clear_unit_shell_cache()
    for got in runs:
        for a, b in zip(got, ref):
            for key in ("B_sugi", "Bk_raw", "Shot_noise"):
                assert rel_err(a[key], b[key]) < 1e-6, key
            assert rel_err(a["SN_terms"]["SN3_FFT"], b["SN_terms"]["SN3_FFT"]) < 1e-6


def test_two_streams_match_serial():
    """Two data vectors queued on two CUDA streams (each with its own library
    context, so they run concurrently) equal the same vectors computed one by
    one on the default stream."""
    import torch
    from cosmonpc_b200 import api
    from cosmonpc_b200.mocks import lognormal_box

    kw = dict(nmesh=64, boxsize=800.0, sampler="pcs", interlaced=True, k_min=0.01, k_max=0.11, k_bins=8,
              angu_configs=[(0, 0, 0), (2, 0, 2)], data_vector_mode="full", shotnoise_mode="both",
              precision="f32")
    cats = [torch.from_numpy(lognormal_box(150000, 800.0, 70 + i)).cuda() for i in range(2)]
    ref = [api.bk_sugi_box_vector(c, None, **kw) for c in cats]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for s in streams:
        s.wait_stream(torch.cuda.current_stream())
    fins = []
    for c, s in zip(cats, streams):
        with torch.cuda.stream(s):
            fins.append(api.bk_sugi_box_vector(c, None, deferred=True, **kw))
    got = [f() for f in fins]
    for g, r in zip(got, ref):
        for a, b in zip(g, r):
            for key in ("B_sugi", "Bk_raw", "Shot_noise"):
                assert rel_err(a[key], b[key]) < 1e-6, key
