"""cosmonpc_b200 -- B200-native drop-in for CosmoNPC's mesh-estimator path.

``run_stats(config)`` takes the reference's config dict and writes the same
``.npy`` result dictionaries; the work runs in hand-written sm_100a kernels and
cuFFT (libcosmonpc_b200.so, C ABI in include/cosmonpc_b200.h).
"""
from .task_executor import run_stats  # noqa: F401

__all__ = ["run_stats"]
