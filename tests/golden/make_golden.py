"""Generate the golden vectors in this folder by running the reference itself.

Run in a container that holds the reference sources (default
/root/reference/src, override with COSMONPC_REFERENCE_SRC):

    python tests/golden/make_golden.py

Each case of ``cases.py`` is run through the reference's own ``run_stats`` with
single-rank stand-ins for mpi4py / numexpr / pmesh (``ref_shims.py``); the
numeric keys of the saved result dict are stored as ``<case>.npz`` together with
the catalog checksums.
"""
from __future__ import annotations

import copy
import glob
import logging
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from cases import CASES, SURVEY_CASES, build_case, flatten_result  # noqa: E402
from ref_shims import import_reference  # noqa: E402


def main(names=None):
    te = import_reference()
    logging.disable(logging.INFO)
    # catalogs live in a folder named "golden": the bispectrum output file name
    # carries the catalog's parent folder name (task_executor.py:305-309)
    work = os.path.join(tempfile.mkdtemp(prefix="cnpc_golden_"), "golden")
    for name, _, _ in CASES + SURVEY_CASES:
        if names and name not in names:
            continue
        cfg, sums = build_case(name, work)
        te.run_stats(copy.deepcopy(cfg))
        files = glob.glob(os.path.join(cfg["output_dir"], "*.npy"))
        assert len(files) == 1, files
        res = np.load(files[0], allow_pickle=True).item()
        flat = flatten_result(res)
        flat.update({"checksum." + k: np.float64(v) for k, v in sums.items()})
        flat["output_name"] = np.array(os.path.basename(files[0]))
        np.savez(os.path.join(HERE, name + ".npz"), **flat)
        print("wrote", name, sorted(flat))


if __name__ == "__main__":
    main(sys.argv[1:] or None)
