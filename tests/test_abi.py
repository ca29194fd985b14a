"""The C-ABI library loads and exports every declared entry point (CPU only: no
compute call is made)."""
import ctypes
import os
import re

import pytest

from slm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            text = open(os.path.join(ROOT, "include", h)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(slm_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        from slm_b200 import build
        build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_every_declared_symbol_exported(lib):
    declared = _declared()
    assert "slm_integrate_fields" in declared
    for name in declared:
        assert hasattr(lib, name), name


def test_bindings_cover_header():
    assert _declared() == set(_lib.SIGNATURES)


def test_version_and_error_strings(lib):
    L = _lib.load()
    assert b"sm_100a" in L.slm_version()
    assert L.slm_last_error() is not None
    assert L.slm_fields_workspace_words() >= 3


def test_bad_arguments_rejected_without_device():
    """Argument checks run on the host before any CUDA call."""
    from slm_b200.params import SlmParams
    L = _lib.load()
    p = SlmParams()  # zero grid -> rejected
    rc = L.slm_integrate_fields(_lib.sref(p), None, None, None, None, None, None, None, None, None)
    assert rc == _lib.SLM_ERR_ARGS
    assert b"grid too small" in L.slm_last_error()
