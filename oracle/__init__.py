"""Oracle: CPU restatement of CosmoNPC's mesh-estimator path.

TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference arm may import anything here, and only
as the checker or as the timed CPU baseline.  The product package
``cosmonpc_b200`` never imports it and has no CPU fallback.

Pinning: the restatement is checked against golden vectors in ``tests/golden``
that ``tests/golden/make_golden.py`` produced by running the unmodified
reference estimator code (src/cosmonpc/*.py) through single-rank stand-ins for
mpi4py, numexpr and pmesh.  The pmesh stand-in (``pmesh_lite``) is itself a
restatement of pmesh's published conventions, so parity at the pmesh boundary
(window node placement, k-vector formula) is unpinned by any reference test.
"""
