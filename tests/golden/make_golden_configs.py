"""Golden vectors of the benchmark workloads at their own sizes (``configs.py``),
made by running the reference itself.

Run in a container that holds the reference sources (default
/root/reference/src, override with COSMONPC_REFERENCE_SRC):

    python tests/golden/make_golden_configs.py [name ...]

Each case of ``configs.CONFIG_CASES`` goes through the reference's own
``run_stats`` with the single-rank stand-ins of ``ref_shims.py`` (pmesh's paint
and FFTs restated on numpy/scipy, FP64 complex128 fields as the reference holds
them); the numeric keys of the saved result dict are stored as
``cfg_<name>.npz`` with the catalog checksums.  The 256^3 full data vectors
take several minutes and ~30 GB of host memory each.
"""
from __future__ import annotations

import copy
import glob
import logging
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from cases import flatten_result  # noqa: E402
from configs import CONFIG_CASES, build_config_case  # noqa: E402
from ref_shims import import_reference  # noqa: E402


def main(names=None):
    te = import_reference()
    logging.disable(logging.INFO)
    work = os.path.join(tempfile.mkdtemp(prefix="cnpc_golden_cfg_"), "golden")
    for name in CONFIG_CASES:
        if names and name not in names:
            continue
        t0 = time.perf_counter()
        cfg, sums = build_config_case(name, work)
        te.run_stats(copy.deepcopy(cfg))
        files = glob.glob(os.path.join(cfg["output_dir"], "*.npy"))
        assert len(files) == 1, files
        res = np.load(files[0], allow_pickle=True).item()
        flat = flatten_result(res)
        flat.update({"checksum." + k: np.float64(v) for k, v in sums.items()})
        flat["output_name"] = np.array(os.path.basename(files[0]))
        np.savez(os.path.join(HERE, "cfg_" + name + ".npz"), **flat)
        print("wrote cfg_%s in %.0f s" % (name, time.perf_counter() - t0), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or None)
