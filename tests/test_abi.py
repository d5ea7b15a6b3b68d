"""The C-ABI library loads and exports every entry point its header
declares (no device needed; nothing here computes)."""
import os
import re

import pytest

import plastimatch_b200 as P

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "plastimatch_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b200bsp_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_functions():
    names = declared_functions()
    assert "b200bsp_create" in names and "b200bsp_score_mse" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    L = P.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(P._SIGS)


def test_version_string():
    assert b"sm_100a" in P.lib().b200bsp_version()


def test_null_arguments_are_rejected_without_crash():
    L = P.lib()
    assert L.b200bsp_create(None, None, None, None, None) == -1
    assert L.b200bsp_destroy(None) == 0
    assert L.b200bsp_score_mse(None, None, None, None, None) == -1
    assert b"null" in L.b200bsp_last_error(None)


def test_reference_side_adapter_links():
    """The reference-side drop-in (oracle/ref/b200_adapter.cxx) resolves
    every symbol against the reference build and this library."""
    import ctypes
    import oracle as O
    if not O.adapter_available():
        pytest.skip("reference-side adapter not built")
    lib = ctypes.CDLL(O.ADAPTER_SO, mode=ctypes.RTLD_GLOBAL)
    assert hasattr(lib, "adapter_compare")
