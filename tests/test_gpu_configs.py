"""The benchmark workloads at their own sizes on the GPU (through the C ABI),
against golden vectors of the reference itself (``golden/configs.py``,
``golden/make_golden_configs.py``).

Workloads: pk 64^3 (1e5 particles), bk_sugi diagonal 128^3 (1e6; (000),
(202), (110)), bk_sugi full 256^3 (4e6; (000), (202), all 400 entries of each
data vector, shot noise "both"), the survey cross workload at 256^3 with a
tenth of its catalogs (pk [0,2,4], bk aab (000) and (202)), and one mock of
each batched-mocks shape class (128^3, 192^3, 256^3).

Bar: every multipole within 1e-8 (FP64 drop-in) or 1e-5 (FP32 fields with
FP64 accumulation) of its max |value| over the bins, mode counts bit for bit.
With CNPC_PARITY_REPORT=<path> each case appends its per-key errors to that
file as one JSON line.
"""
import copy
import os

import numpy as np
import pytest

from cases import flatten_result
from configs import CONFIG_CASES, build_config_case
from conftest import GOLDEN, parity_report, rel_err

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-8, "f32": 1e-5}


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    # the bispectrum file name carries the catalog's parent folder name
    return str(tmp_path_factory.mktemp("configs") / "golden")


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("name", list(CONFIG_CASES))
def test_config_case_matches_reference(name, precision, workdir, tmp_path):
    import cosmonpc_b200

    gold = np.load(os.path.join(GOLDEN, "cfg_%s.npz" % name))
    cfg, sums = build_config_case(name, workdir)
    for k, v in sums.items():  # the regenerated catalogs are the ones the reference ran on
        assert float(gold["checksum." + k]) == pytest.approx(v, rel=1e-13, abs=0.0), k
    cfg = copy.deepcopy(cfg)
    cfg["precision"] = precision
    cfg["output_dir"] = str(tmp_path / ("out_" + precision))
    path = cosmonpc_b200.run_stats(cfg)
    assert os.path.basename(path) == str(gold["output_name"])
    got = flatten_result(np.load(path, allow_pickle=True).item())
    keys = {k for k in gold.files if not k.startswith("checksum") and k != "output_name"}
    assert keys <= set(got), keys - set(got)
    errs = {}
    for k in sorted(keys):
        if k in ("k_num", "nmodes"):
            np.testing.assert_array_equal(got[k], gold[k])
        else:
            errs[k] = rel_err(got[k], gold[k])
    parity_report(name, precision, errs)
    bad = {k: e for k, e in errs.items() if not e < TOL[precision]}
    assert not bad, (bad, errs)
