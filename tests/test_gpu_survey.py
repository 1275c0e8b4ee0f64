"""Survey path on the GPU (through the C ABI) against the oracle and the
reference's own golden vectors.

Tolerances as for the box (conftest.tol): FP64 to 1e-8 of each multipole's
max |value|, FP32 to 1e-5, mode counts bit for bit; stage checks against the
oracle at FP64 rounding level.
"""
import copy
import os

import numpy as np
import pytest

from cases import SURVEY_CASES, build_case, flatten_result
from conftest import GOLDEN, parity_report, rel_err, tol

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-8, "f32": 1e-5}
SURVEY = dict(column_names=["RA", "DEC", "Z", "WEIGHT_FKP", "WEIGHT_SYSTOT", "WEIGHT_NOZ", "WEIGHT_CP", "NZ"],
              cosmology={"h": 0.6766, "Omega0": 0.31})


def _mixed_type_catalog(path, n=5000, seed=3):
    """A catalog whose weight columns use the integer and float32 FITS types
    (angles and redshifts stay float64, as in survey catalogs)."""
    from cosmonpc_b200 import fits, mocks

    d, _ = mocks.survey_catalogs(n, 1000, seed, boss_weights=True)
    cols = {"RA": d["RA"], "DEC": d["DEC"], "ID": np.arange(len(d["Z"]), dtype=np.int64),
            "Z": d["Z"], "NZ": d["NZ"].astype(np.float32), "WEIGHT_FKP": d["WEIGHT_FKP"],
            "WEIGHT_SYSTOT": d["WEIGHT_SYSTOT"].astype(np.float32),
            "WEIGHT_NOZ": d["WEIGHT_NOZ"].astype(np.int32), "WEIGHT_CP": d["WEIGHT_CP"].astype(np.int16)}
    fits.write_table(path, cols)
    return path


@pytest.mark.parametrize("scheme,ctype,zr", [("boss", "data", (0.42, 0.58)), ("eboss", "data", None),
                                             (None, "randoms", (0.45, 0.5)), ("boss", "randoms", None)])
def test_catalog_decode_matches_oracle(tmp_path, scheme, ctype, zr):
    from cosmonpc_b200 import survey
    from oracle.survey import read_catalog as oracle_read

    path = _mixed_type_catalog(str(tmp_path / "cat.fits"))
    plan = {"scheme": scheme, "name_alias": None}
    cat = survey.read_catalog(path, SURVEY["column_names"], zr, plan, ctype, SURVEY["cosmology"])
    ref, _ = oracle_read(path, SURVEY["column_names"], zr, plan, ctype, SURVEY["cosmology"], "particle")
    assert cat.n == len(ref["w"])
    pos = cat.pos.cpu().numpy()
    assert np.max(np.abs(pos - ref["pos"])) < 1e-12 * np.max(np.abs(ref["pos"]))
    np.testing.assert_array_equal(cat.w.cpu().numpy(), ref["w"])
    np.testing.assert_array_equal(cat.wfkp.cpu().numpy(), ref["wfkp"])
    np.testing.assert_array_equal(cat.nz.cpu().numpy(), ref["nz"])


def test_catalog_errors_match_reference(tmp_path):
    from cosmonpc_b200 import survey

    path = _mixed_type_catalog(str(tmp_path / "cat.fits"))
    cols = SURVEY["column_names"]
    with pytest.raises(ValueError, match="Alias WX not found"):
        survey.read_catalog(path, cols, None, {"scheme": None, "name_alias": "WX"}, "data", SURVEY["cosmology"])
    with pytest.raises(ValueError, match="both a scheme and an alias"):
        survey.read_catalog(path, cols, None, {"scheme": "boss", "name_alias": "NZ"}, "data", SURVEY["cosmology"])
    with pytest.raises(ValueError, match="WEIGHT_FKP column is missing"):
        survey.read_catalog(path, [c for c in cols if c != "WEIGHT_FKP"], None,
                            {"scheme": None, "name_alias": None}, "data", SURVEY["cosmology"])
    with pytest.raises(ValueError, match="NZ column is missing"):
        survey.read_catalog(path, [c for c in cols if c != "NZ"], None, {"scheme": None, "name_alias": None},
                            "data", SURVEY["cosmology"], "particle")
    with pytest.raises(NotImplementedError):
        survey.read_catalog(str(tmp_path / "x.npy"), cols, None, {"scheme": None, "name_alias": None}, "data",
                            SURVEY["cosmology"])


def test_particle_sums_and_boxcenter(tmp_path):
    from cosmonpc_b200 import survey
    from oracle import angular
    from oracle.survey import read_catalog as oracle_read

    path = _mixed_type_catalog(str(tmp_path / "cat.fits"), n=20000)
    plan = {"scheme": "boss", "name_alias": None}
    cat = survey.read_catalog(path, SURVEY["column_names"], None, plan, "data", SURVEY["cosmology"])
    ref, bc = oracle_read(path, SURVEY["column_names"], None, plan, "data", SURVEY["cosmology"], "particle")
    s = survey.ParticleSums(cat, L=2)
    w, f, nz, pos = ref["w"], ref["wfkp"], ref["nz"], ref["pos"]
    assert s.w_wfkp == pytest.approx(np.sum(w * f), rel=1e-13)
    assert s.w == pytest.approx(np.sum(w), rel=1e-13)
    assert s.I_sum == pytest.approx(np.sum(w * nz * f * f), rel=1e-13)
    assert s.N_sum == pytest.approx(np.sum((w * f) ** 2), rel=1e-13)
    assert s.I33 == pytest.approx(np.sum(nz ** 2 * w ** 2 * f ** 3), rel=1e-13)
    u = pos / np.linalg.norm(pos, axis=1, keepdims=True)
    for M in range(3):
        ref_s = np.sum((w * f) ** 3 * np.conj(angular.ylm_function(2, M, True)(u[:, 0], u[:, 1], u[:, 2])))
        assert abs(s.S_LM[M] - ref_s) < 1e-12 * max(1.0, abs(ref_s))
    np.testing.assert_allclose(survey.boxcenter_of(s), bc, rtol=0, atol=1e-12 * np.max(np.abs(bc)))


@pytest.mark.parametrize("sampler,interlaced", [("cic", True), ("pcs", True), ("tsc", False)])
def test_interlaced_field_real_and_imaginary_parts(tmp_path, sampler, interlaced):
    """Re and Im of the painted complex field against the oracle's c2c version."""
    from cosmonpc_b200 import survey
    from oracle.box import paint_field

    path = _mixed_type_catalog(str(tmp_path / "cat.fits"), n=20000)
    plan = {"scheme": None, "name_alias": None}
    cat = survey.read_catalog(path, SURVEY["column_names"], None, plan, "data", SURVEY["cosmology"])
    bc = survey.boxcenter_of(survey.ParticleSums(cat))
    w = cat.paint_weights()
    n, L = 32, 1000.0
    F = survey.paint_field([(cat, w, 0.5)], n, L, sampler, interlaced, bc, "f64")
    ref = 0.5 * paint_field(cat.pos.cpu().numpy() - bc, w.cpu().numpy(), n, L, sampler, interlaced)
    re = F.re.cpu().numpy()
    assert np.max(np.abs(re - ref.real)) < 1e-12 * np.max(np.abs(ref.real))
    if interlaced:
        im = F.im.cpu().numpy()
        assert np.max(np.abs(ref.imag)) > 1e-3 * np.max(np.abs(ref.real))  # the residue is real
        assert np.max(np.abs(im - ref.imag)) < 1e-12 * np.max(np.abs(ref.real))
    else:
        assert F.im is None


@pytest.mark.parametrize("l,m,conj", [(2, 0, False), (2, 1, True), (4, 3, False)])
def test_xspace_harmonic_matches_oracle(l, m, conj):
    import torch
    from cosmonpc_b200 import _lib, angular as dang, engine
    from oracle import angular
    from oracle.survey import xgrid

    n, L = 24, 700.0
    bc = np.array([-900.0, 310.0, 440.0])
    rng = np.random.default_rng(l * 10 + m)
    fr, fi = rng.standard_normal((n, n, n)), rng.standard_normal((n, n, n))
    ctx = _lib.Context.get()
    out = torch.empty((2, n, n, n), dtype=torch.float64, device="cuda")
    ctx.xspace_harmonic(_lib.F64, n, L, bc, torch.from_numpy(fr).cuda(), torch.from_numpy(fi).cuda(),
                        dang.harmonic(l, m, True), conj, 1.0, out[0], out[1])
    y = angular.ylm_function(l, m, True)(*xgrid(n, L, bc))
    ref = (fr + 1j * fi) * (np.conj(y) if conj else y)
    got = out[0].cpu().numpy() + 1j * out[1].cpu().numpy()
    assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))


def _run(cfg, precision, tmp_path):
    import cosmonpc_b200

    cfg = copy.deepcopy(cfg)
    cfg["precision"] = precision
    cfg["output_dir"] = str(tmp_path / ("out_" + precision))
    path = cosmonpc_b200.run_stats(cfg)
    return np.load(path, allow_pickle=True).item(), os.path.basename(path)


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name", [c[0] for c in SURVEY_CASES])
def test_survey_golden_case(name, precision, tmp_path):
    cfg, _ = build_case(name, str(tmp_path / "golden"))
    gold = np.load("%s/%s.npz" % (GOLDEN, name))
    res, fname = _run(cfg, precision, tmp_path)
    assert fname == str(gold["output_name"])
    got = flatten_result(res)
    keys = {k for k in gold.files if not k.startswith("checksum") and k != "output_name"}
    assert keys <= set(got), keys - set(got)
    errs = {k: rel_err(got[k], gold[k]) for k in sorted(keys) if k not in ("k_num", "nmodes")}
    for k in ("k_num", "nmodes"):
        if k in keys:
            np.testing.assert_array_equal(got[k], gold[k])
    parity_report(name, precision, errs)
    bad = {k: e for k, e in errs.items() if not e < tol(precision, name, k)}
    assert not bad, (bad, errs)
    assert res["nmesh"] == cfg["nmesh"] and "nyquist_freq" in res
