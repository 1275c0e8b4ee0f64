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
    """Parity tolerance of one output: 1e-8 in FP64; in FP32 1e-5, raised to
    4x the error that single-precision FFTs alone cause on the case (measured
    by tests/golden/make_fp32_conditioning.py) where that is larger."""
    import json

    if precision == "f64":
        return 1e-8
    global _COND
    if _COND is None:
        with open(os.path.join(GOLDEN, "fp32_fft_conditioning.json")) as f:
            _COND = json.load(f)
    return max(1e-5, 4.0 * _COND.get(case, {}).get(key, 0.0))


_COND = None

