import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)
GOLDEN = os.path.join(REPO, "tests", "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")


def rel_err(got, ref):
    """max |got - ref| / max |ref| (the per-multipole criterion of the parity bar)."""
    import numpy as np

    got = np.asarray(got, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(got - ref))) if got.size else 0.0
    return float(np.max(np.abs(got - ref)) / scale)


def tol(precision, case, key):
    """Parity tolerance of one output: 1e-8 of each multipole's max |value| in
    FP64, 1e-5 in FP32 (the parity bar)."""
    return 1e-8 if precision == "f64" else 1e-5


def parity_report(name, precision, errs):
    """With CNPC_PARITY_REPORT=<path>, append a case's per-key errors as one JSON line."""
    import json

    path = os.environ.get("CNPC_PARITY_REPORT")
    if path and errs:
        with open(path, "a") as f:
            f.write(json.dumps({"case": name, "precision": precision, "max": max(errs.values()), "errors": errs})
                    + "\n")
