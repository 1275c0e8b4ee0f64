"""How far single-precision FFTs alone move each golden case's outputs.

The FP32 precision mode computes every transform in FP32.  On small,
ill-conditioned cases (few modes per bin, signal that cancels between modes)
the FFT rounding by itself is already a few 1e-6 of a multipole's maximum, so
the FP32 parity tolerance of a case is set from this measured conditioning:
the oracle is run with its forward and inverse FFTs rounded through complex64
(scipy's pocketfft in single precision), everything else in FP64, and the
error of each output key against the reference's own golden vector is
written to ``fp32_fft_conditioning.json``.

Run from the repository root:  python tests/golden/make_fp32_conditioning.py
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np
import scipy.fft as sfft

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [HERE, os.path.dirname(HERE), ROOT]

from cases import CASES, SURVEY_CASES, build_case, flatten_result  # noqa: E402


def _err(got, ref):
    got = np.asarray(got, dtype=np.complex128)
    ref = np.asarray(ref, dtype=np.complex128)
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    d = float(np.max(np.abs(got - ref))) if got.size else 0.0
    return d / scale if scale else d


def main():
    import oracle.box as ob
    from oracle.driver import run_box
    from oracle.survey import run_survey

    ob._fftn = lambda a: sfft.fftn(np.asarray(a).astype(np.complex64), workers=-1).astype(np.complex128)
    ob._ifftn = lambda a: sfft.ifftn(np.asarray(a).astype(np.complex64), workers=-1).astype(np.complex128)
    out = {}
    tmp = tempfile.mkdtemp()
    for name, _, _ in CASES + SURVEY_CASES:
        cfg, _ = build_case(name, os.path.join(tmp, name))
        gold = np.load(os.path.join(HERE, name + ".npz"))
        got = flatten_result(run_survey(cfg) if name.startswith("sv_") else run_box(cfg))
        keys = [k for k in gold.files if not k.startswith("checksum") and k not in ("output_name", "k_num", "nmodes")
                and gold[k].dtype.kind not in "US"]
        out[name] = {k: float("%.3e" % _err(got[k], gold[k])) for k in sorted(keys)}
        print(name, max(out[name].values()), flush=True)
    with open(os.path.join(HERE, "fp32_fft_conditioning.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
