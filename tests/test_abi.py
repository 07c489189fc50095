"""C-ABI checks that need no GPU: the library loads and exports every declared entry point."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "epb200.h")


def _declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"EPB_API\s+(?:int|const char\*)\s+(epb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = _declared()
    assert "epb_create" in names and "epb_fourier" in names and "epb_eigh_batched" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from epb200 import _lib

    L = _lib.lib()
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"
    # every binding has a declaration
    assert set(_lib.SIGNATURES) <= set(_declared())


def test_version_and_error_string_without_gpu():
    from epb200 import _lib

    L = _lib.lib()
    assert L.epb_version() >= 100
    assert isinstance(L.epb_last_error(), bytes)


def test_create_fails_cleanly_without_gpu():
    """On a machine without a GPU, epb_create reports an error instead of crashing."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    from epb200 import _lib

    h = ctypes.c_void_p()
    st = _lib.lib().epb_create(ctypes.byref(h), 0, None)
    assert st != _lib.EPB_OK
    assert _lib.lib().epb_last_error()


def test_null_ctx_is_rejected():
    from epb200 import _lib

    L = _lib.lib()
    assert L.epb_synchronize(None) == _lib.EPB_ERR_ARG
    assert L.epb_fourier(None, None, 0, 0, None, None, 0, None, 0) == _lib.EPB_ERR_ARG
    assert b"NULL" in L.epb_last_error()
