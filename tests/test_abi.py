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


def test_pair_and_preprocess_arguments_rejected_without_device():
    """Host-side checks of the pair launch, preprocess and seed entry points
    (nothing reaches the device): mismatched direction blocks, a bad upstream
    stride, a bad ROI type, a too-small seed buffer."""
    import numpy as np

    from cases import Case
    L = _lib.load()
    c = Case(nx=20, ny=16, seed=3)
    pd, pu = c.params("INTEGRATE_FIELDS", 1.0), c.params("INTEGRATE_FIELDS", -1.0)
    fake = ctypes.c_void_p(4096)  # never dereferenced: the checks fail first
    bad = c.params("INTEGRATE_FIELDS", -1.0)
    bad.max_n_steps += 1
    rc = L.slm_integrate_fields_pair(_lib.sref(pd), _lib.sref(bad), None, fake, fake, fake, fake, fake,
                                     pd.nxy_padded, fake, None, None, None)
    assert rc == _lib.SLM_ERR_ARGS and b"differ in more than the direction" in L.slm_last_error()
    same = c.params("INTEGRATE_FIELDS", 1.0)
    rc = L.slm_integrate_fields_pair(_lib.sref(pd), _lib.sref(same), None, fake, fake, fake, fake, fake,
                                     pd.nxy_padded, fake, None, None, None)
    assert rc == _lib.SLM_ERR_ARGS  # same sign twice
    rc = L.slm_integrate_fields_pair(_lib.sref(pd), _lib.sref(pu), None, fake, fake, fake, fake, fake,
                                     pd.nxy_padded - 1, fake, None, None, None)
    assert rc == _lib.SLM_ERR_ARGS and b"up_stride" in L.slm_last_error()
    prm = _lib.SlmPreprocessParams(1.0, 0.95, -0.5, 0.0, 2, 1)
    rc = L.slm_preprocess(fake, 7, 10, 10, ctypes.byref(prm), fake, None, None, None, None, None, None, None,
                          None, None, None)
    assert rc == _lib.SLM_ERR_ARGS and b"roi_dtype" in L.slm_last_error()
    mask = np.zeros((6, 5), np.uint8)
    out = np.empty((3, 2), np.float32)
    n = ctypes.c_uint64(0)
    rc = L.slm_create_seeds(mask.ctypes.data, 6, 5, 1, 1, 1, out.ctypes.data, 3, ctypes.byref(n), None)
    assert rc == _lib.SLM_ERR_CAPACITY and n.value == 30


def test_fmm_lengths_arguments_rejected_without_device():
    """slm_fmm_lengths' host checks (nothing reaches the device): an order
    other than 1 or 2, an empty window, a null buffer; no problems is a
    no-op that touches nothing."""
    L = _lib.load()
    fake = ctypes.c_void_p(4096)  # never dereferenced: the checks fail first

    def call(nx=8, ny=8, n=1, order=2, val=fake):
        return L.slm_fmm_lengths(fake, fake, nx, ny, 1, fake, fake, fake, n, 64, order, 1.0, val, fake, fake,
                                 fake, fake, fake, fake, fake, fake, None)
    assert call(order=3) == _lib.SLM_ERR_ARGS and b"order" in L.slm_last_error()
    assert call(nx=0) == _lib.SLM_ERR_ARGS and b"window" in L.slm_last_error()
    assert call(val=None) == _lib.SLM_ERR_ARGS and b"null" in L.slm_last_error()
    assert call(n=0, val=None) == _lib.SLM_OK
