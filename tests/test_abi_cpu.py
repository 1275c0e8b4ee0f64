"""The C-ABI library builds, loads on a machine without a GPU, and exports every
entry point declared in include/*.h (no compute calls here)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import REPO


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(cnpc_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from cosmonpc_b200 import build

    lib_path = build.build()
    lib = ctypes.CDLL(lib_path)
    names = declared_symbols()
    assert len(names) >= 12
    for name in sorted(names):
        assert hasattr(lib, name), name


def test_binding_covers_exports():
    from cosmonpc_b200 import _lib

    assert set(_lib.EXPORTED) <= declared_symbols()
    assert set(_lib._SIGS) == set(_lib.EXPORTED)


def test_status_strings_and_context_without_gpu():
    from cosmonpc_b200 import _lib

    lib = _lib.load()
    assert lib.cnpc_version() >= 100
    assert lib.cnpc_status_string(_lib.CNPC_EINVAL) == b"invalid argument"
    h = ctypes.c_void_p()
    # no CUDA device in this container: creation must fail cleanly, not crash
    import torch

    if not torch.cuda.is_available():
        assert lib.cnpc_ctx_create(ctypes.byref(h), 0) == _lib.CNPC_ECUDA


def test_struct_layouts_match_header():
    from cosmonpc_b200 import _lib
    from cosmonpc_b200.angular import Harmonic

    assert ctypes.sizeof(Harmonic) == 4 + 4 + 8 + 9 * 8 + 8 + 8
    assert ctypes.sizeof(_lib.ShellItem) == 5 * 4


def test_device_path_fails_loudly_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from cosmonpc_b200 import _lib

    with pytest.raises(RuntimeError):
        _lib.Context.get()


def test_survey_struct_layouts_match_c_compiler(tmp_path):
    """sizeof / offsetof of the survey structs as gcc lays them out from the header."""
    import subprocess

    from cosmonpc_b200 import _lib

    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "cosmonpc_b200.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(cnpc_column), sizeof(cnpc_catalog_spec),'
        ' sizeof(cnpc_operand), offsetof(cnpc_catalog_spec, weight_rule), offsetof(cnpc_catalog_spec, h),'
        ' offsetof(cnpc_operand, comp), sizeof(cnpc_harmonic)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    from cosmonpc_b200.angular import Harmonic

    want = [ctypes.sizeof(_lib.Column), ctypes.sizeof(_lib.CatalogSpec), ctypes.sizeof(_lib.Operand),
            _lib.CatalogSpec.weight_rule.offset, _lib.CatalogSpec.h.offset, _lib.Operand.comp.offset,
            ctypes.sizeof(Harmonic)]
    assert got == want
