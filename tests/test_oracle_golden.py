"""The oracle restatement against golden vectors produced by the reference itself."""
import numpy as np
import pytest

from cases import CASES, SURVEY_CASES, build_case, flatten_result
from conftest import GOLDEN, rel_err

NAMES = [c[0] for c in CASES]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(name, tmp_path):
    from oracle.driver import run_box

    cfg, sums = build_case(name, str(tmp_path / "golden"))
    gold = np.load("%s/%s.npz" % (GOLDEN, name))
    for letter, s in sums.items():
        assert s == pytest.approx(float(gold["checksum." + letter]), rel=0, abs=1e-6), \
            "synthetic catalog generator drifted"
    got = flatten_result(run_box(cfg))
    ref_keys = {k for k in gold.files if not k.startswith("checksum") and k != "output_name"}
    assert set(got) == ref_keys
    for k in sorted(ref_keys):
        if k in ("k_num", "nmodes"):
            np.testing.assert_array_equal(got[k], gold[k])
        else:
            assert rel_err(got[k], gold[k]) < 1e-11, k


SURVEY_NAMES = [c[0] for c in SURVEY_CASES]


@pytest.mark.parametrize("name", SURVEY_NAMES)
def test_survey_oracle_matches_reference_golden(name, tmp_path):
    """The survey restatement (complex fields, comoving distance by 2F1) against the reference."""
    from oracle.survey import run_survey

    cfg, sums = build_case(name, str(tmp_path / "golden"))
    gold = np.load("%s/%s.npz" % (GOLDEN, name))
    for key, s in sums.items():
        assert s == pytest.approx(float(gold["checksum." + key]), rel=0, abs=1e-6), \
            "synthetic catalog generator drifted"
    got = flatten_result(run_survey(cfg))
    ref_keys = {k for k in gold.files if not k.startswith("checksum") and k != "output_name"
                and gold[k].dtype.kind not in "US"}
    assert ref_keys <= set(got), ref_keys - set(got)
    for k in sorted(ref_keys):
        if k in ("k_num", "nmodes"):
            np.testing.assert_array_equal(got[k], gold[k])
        else:
            assert rel_err(got[k], gold[k]) < 1e-11, (k, rel_err(got[k], gold[k]))
