"""The allocation-free contraction entry point against the regular one.

cnpc_contract_gram_noalloc is for callers that cannot let the library call
cudaMalloc (an application whose own memory pool owns the device, or one that
cannot take the synchronisation cudaFree may cause); it keeps its partial sums
in a fixed array in the library's device memory.  This file is collected last
so that a run stopping at the first failure has already run every other test;
it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-8, "f32": 1e-5}


# (rows, columns): columns a run of the rows (staged once), columns outside
# the rows (staged separately), and a 40 x 24 FP32 window (41 staged rows),
# where the fixed array, not the SM count, bounds the number of blocks
CASES = [("f32", list(range(40)), list(range(5, 25))), ("f32", list(range(20)), list(range(20))),
         ("f32", list(range(16)), list(range(20, 28))), ("f32", list(range(40)), list(range(16, 40))),
         ("f64", list(range(40)), list(range(5, 25))), ("f64", list(range(12)), list(range(7))),
         ("f64", list(range(12)), list(range(30, 37)))]


@pytest.mark.parametrize("precision,a,b", CASES)
def test_noalloc_matches_gram_twice(precision, a, b):
    import torch

    from cosmonpc_b200 import _lib, engine

    code, rdt, _ = engine.PRECISION[precision]
    ctx = _lib.Context.get()
    lib = _lib.load()
    n = 64
    ncell = n ** 3
    na, nb = len(a), len(b)
    gen = torch.Generator(device="cuda").manual_seed(7 + na + 100 * b[0])
    fields = torch.randn((48, ncell), dtype=rdt, device="cuda", generator=gen)
    G = torch.randn(ncell, dtype=rdt, device="cuda", generator=gen)
    ref = torch.empty((na, nb), dtype=torch.float64, device="cuda")
    ctx.gram(code, ncell, G, fields, ncell, a, b, ref)
    aa = (ctypes.c_int * na)(*a)
    bb = (ctypes.c_int * nb)(*b)
    stream = ctx.stream()
    for _ in range(2):  # the shared array keeps the previous call's contents
        out = torch.full((na, nb), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.cnpc_contract_gram_noalloc(code, ncell, ctypes.c_void_p(G.data_ptr()),
                                            ctypes.c_void_p(fields.data_ptr()), ncell, aa, na, bb, nb,
                                            ctypes.c_void_p(out.data_ptr()), stream)
        assert st == _lib.CNPC_OK
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy()) < TOL[precision]


def test_noalloc_rejects_oversized_calls():
    import torch

    from cosmonpc_b200 import _lib

    lib = _lib.load()
    x = torch.zeros(1024, dtype=torch.float32, device="cuda")
    out = torch.zeros(64 * 32, dtype=torch.float64, device="cuda")
    a = (ctypes.c_int * 64)(*([0] * 64))
    b = (ctypes.c_int * 32)(*([0] * 32))
    st = lib.cnpc_contract_gram_noalloc(_lib.F32, 1024, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                        1024, a, 64, b, 32, ctypes.c_void_p(out.data_ptr()), None)
    assert st == _lib.CNPC_EINVAL
