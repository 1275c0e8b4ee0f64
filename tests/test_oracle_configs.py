"""The oracle against golden vectors of the reference itself at the benchmark
workloads' own sizes (``golden/configs.py``): pk 64^3, bk_sugi diagonal 128^3
((000), (202), (110)), one 128^3 mock (pk and bk (000)), and the 256^3 full
data vectors on a fixed subset of (k1, k2) entries (every shot-noise term
except SN3_FFT in full; the triple sums of bins 0, 9 and 19)."""
import numpy as np
import pytest

from configs import CONFIG_CASES, build_config_case
from conftest import GOLDEN, rel_err

CHEAP = ["c1_pk_64", "c2_bk_diag_128_000", "c2_bk_diag_128_202", "c2_bk_diag_128_110", "c5_mock_128_pk",
         "c5_mock_128_bk000"]
SUBSET = [0, 9, 19]


def _oracle(cfg, bins=None):
    from oracle import box as obox
    from oracle.driver import read_box_catalog

    pos, w = read_box_catalog(cfg["catalogs"]["data_a"], cfg["column_names"])
    n, L = int(cfg["nmesh"][0]), float(cfg["boxsize"][0])
    field = obox.paint_field(pos, w, n, L, cfg["sampler"], cfg["interlaced"])
    NZ = w.sum() / L ** 3
    if cfg["statistic"] == "pk":
        return obox.pk_box(field, None, "auto", n, L, cfg["k_min"], cfg["k_max"], cfg["k_bins"], cfg["poles"],
                           cfg["sampler"], cfg["interlaced"], cfg["rsd"], NZ)
    return obox.bk_sugi_box(field, None, None, "auto", "aaa", n, L, cfg["k_min"], cfg["k_max"], cfg["k_bins"],
                            list(cfg["angu_config"]), cfg["sampler"], cfg["data_vector_mode"],
                            cfg["shotnoise_mode"], {"a": len(pos)}, {"a": NZ}, bins=bins)


def _flat(res):
    from cases import flatten_result

    return flatten_result(res)


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("ocfg") / "golden")


@pytest.mark.parametrize("name", CHEAP)
def test_oracle_matches_reference_at_size(name, workdir):
    gold = np.load("%s/cfg_%s.npz" % (GOLDEN, name))
    cfg, sums = build_config_case(name, workdir)
    for k, v in sums.items():
        assert float(gold["checksum." + k]) == pytest.approx(v, rel=1e-13, abs=0.0), k
    got = _flat(_oracle(cfg))
    for k in got:
        if k in ("k_num", "nmodes"):
            np.testing.assert_array_equal(got[k], gold[k])
        else:
            assert rel_err(got[k], gold[k]) < 1e-11, (k, rel_err(got[k], gold[k]))


def test_oracle_matches_reference_256_full_subset(workdir):
    """256^3 full data vectors, both configurations: the entries of bins 0, 9 and
    19 of every pair-sum matrix, every analytic shot-noise term in full."""
    from oracle import box as obox
    from oracle.driver import read_box_catalog

    cfg0, sums = build_config_case("c3_bk_full_256_000", workdir)
    pos, w = read_box_catalog(cfg0["catalogs"]["data_a"], cfg0["column_names"])
    n, L = 256, 2000.0
    field = obox.paint_field(pos, w, n, L, "pcs", True)
    NZ = w.sum() / L ** 3
    idx = np.ix_(SUBSET, SUBSET)
    for name in ("c3_bk_full_256_000", "c3_bk_full_256_202"):
        gold = np.load("%s/cfg_%s.npz" % (GOLDEN, name))
        assert float(gold["checksum.a"]) == pytest.approx(sums["a"], rel=1e-13, abs=0.0)
        cfg, _ = build_config_case(name, workdir)
        got = _flat(obox.bk_sugi_box(field, None, None, "auto", "aaa", n, L, 0.01, 0.20, 20, cfg["angu_config"],
                                     "pcs", "full", "both", {"a": len(pos)}, {"a": NZ}, bins=SUBSET))
        for k, v in got.items():
            if k in ("k_num", "nmodes"):
                np.testing.assert_array_equal(v, gold[k])
            elif np.ndim(v) == 2:
                assert rel_err(v[idx], gold[k][idx]) < 1e-11, (name, k)
            else:
                assert rel_err(v, gold[k]) < 1e-11, (name, k)
