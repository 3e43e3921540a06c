"""The C ABI library loads and exports every entry point include/pamo_b200.h
declares; without a GPU the entry points report an error instead of running
anything on the host."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "pamo_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?(?:int|void|char|long long)\s*\*?\s*(pamo_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("pamo_ctx_create", "pamo_free_forward", "pamo_stage2_run", "pamo_simplify"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from pamo_b200 import _lib

    L = _lib.lib()
    for n in declared_functions():
        assert hasattr(L, n), n
    assert set(_lib.SIGNATURES) <= set(declared_functions())


def test_status_strings():
    from pamo_b200 import _lib

    L = _lib.lib()
    assert L.pamo_status_string(0) == b"ok"
    assert L.pamo_status_string(5) == b"no CUDA device"
    assert L.pamo_version() >= 100


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pamo_b200 import _lib

    h = ctypes.c_void_p()
    rc = _lib.lib().pamo_ctx_create(0, ctypes.byref(h))
    assert rc == 5 and not h.value
    with pytest.raises(_lib.PamoError):
        _lib.Context(0)


def test_invalid_arguments_rejected():
    from pamo_b200 import _lib

    L = _lib.lib()
    assert L.pamo_ctx_destroy(None) == 1
    assert L.pamo_stage2_offset(None, None) == 1
