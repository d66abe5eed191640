"""CPU checks of the C-ABI boundary: the library loads without a GPU and
exports every entry point that include/tapas_b200.h declares; context
creation without a GPU fails with a status code, not an abort."""
import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "tapas_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tapas_b200_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def libpath(tb):
    from importlib import import_module
    build = import_module("tapas_reduce_b200.build")
    return build.build()


def test_header_declares_entry_points():
    names = declared_functions()
    assert "tapas_b200_partition" in names and "tapas_b200_evaluate" in names
    assert len(names) >= 20


def test_library_exports_all_declared(libpath, tb):
    L = ctypes.CDLL(str(libpath))
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(tb._lib.EXPORTS) <= set(declared_functions())


def test_ctx_create_without_gpu_is_a_status(libpath, tb):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(tb.TapasError) as e:
        tb.Context(0)
    assert e.value.code in (-2, -1)
