"""The preprocess oracle against the reference's own Python (CPU only).

Pins: tests/golden/preprocess_*.npz, made by running the reference's
Preprocess.find_blockages / conditioned_gradient_vector_field / mask_nan_uv
(tests/golden/make_preprocess_golden.py).  Where the reference checkout is
present, further seeded cases run the reference directly.
"""
import glob
import os
import sys

import numpy as np
import pytest

import dtm_preprocess as D
from slm_b200 import _lib

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("uv_array", "slope_array", "uv_mask_array", "blockages_array", "blocked_neighbors_array",
        "where_looped_array", "roi_gradx_array", "roi_grady_array")


def _files():
    f = sorted(glob.glob(os.path.join(GOLDEN, "preprocess_*.npz")))
    assert f, "preprocess golden fixtures missing"
    return f


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype == bool:
        return np.array_equal(a, b)
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


def run_oracle(g):
    return D.conditioned_uv(g["roi"], float(g["pixel_size"]), int(g["pad_width"]),
                            do_normalize_speed=bool(g["do_normalize_speed"]))


@pytest.mark.parametrize("path", _files())
def test_oracle_matches_reference_golden(path):
    g = np.load(path)
    r = run_oracle(g)
    for k in KEYS:
        assert _same(r[k], g[k]), k
    assert r["n_loops"] == int(g["n_loops"])


def test_golden_cases_exercise_every_fix():
    total = {"loops": 0, "blk": 0, "nbr": 0, "nan": 0, "f64": 0, "raw": 0}
    for path in _files():
        g = np.load(path)
        total["loops"] += int(g["n_loops"])
        total["blk"] += int(np.count_nonzero(g["blockages_array"]))
        total["nbr"] += int(np.count_nonzero(g["blocked_neighbors_array"]))
        total["nan"] += int(g["uv_mask_array"].sum())
        total["f64"] += g["roi"].dtype == np.float64
        total["raw"] += not bool(g["do_normalize_speed"])
    assert all(v > 0 for v in total.values()), total


def test_flow_vector_priority():
    assert D.flow_vector(16 | 1) == (-1, -1)
    assert D.flow_vector(2 | 8) == (1, 0)
    assert D.flow_vector(8) == (0, 1)
    assert D.flow_vector(0) == (0, 0)


def test_vectorised_break_equals_scalar_scan():
    rng = np.random.default_rng(4)
    roi = rng.standard_normal((40, 30)).astype(np.float32)
    roi[rng.random(roi.shape) < 0.1] = np.nan
    roi[5, 5:8] = np.inf
    marked = rng.random(roi.shape) < 0.5
    fix, xs, ys, bu, bv = D.break_vectors(roi, marked)
    assert fix.sum() == xs.size > 0
    for x, y, a, b in zip(xs, ys, bu, bv):
        assert D.break_vector(roi, x, y) == (a, b)


def test_blockage_code_is_diagonal_only():
    roi = np.array([[5.0, 5.0, 5.0], [5.0, 4.0, 5.0], [3.0, 5.0, 5.0]], np.float32)
    c = D.blockage_codes(roi)
    assert c[1, 1] == 32  # the only lower neighbour is at (+x, -y): SE
    roi2 = np.full((3, 3), 5.0, np.float32)
    roi2[1, 1] = 6.0
    roi2[0, 0] = 4.0
    c2 = D.blockage_codes(roi2)
    # every neighbour (5) and the corner (4) is lower: cardinal outflows -> no blockage
    assert c2[1, 1] == 0


def test_reference_direct(reference_dir):
    """Further seeded cases through the reference's own code (needs the checkout)."""
    sys.path.insert(0, GOLDEN)
    try:
        import make_preprocess_golden as M
    finally:
        sys.path.remove(GOLDEN)
    import warnings
    warnings.simplefilter("ignore", DeprecationWarning)
    mod = M.load_reference_preprocess(reference_dir)
    for seed in (31, 32, 33):
        case = dict(nx=23 + seed % 7, ny=29 + seed % 5, seed=seed, pixel_size=1.0 + 0.25 * (seed % 3),
                    pad=seed % 4, noise=0.15, holes=seed % 2 == 0, normalize=seed != 32)
        g = M.run_case(mod, **case)
        r = run_oracle(g)
        for k in KEYS:
            assert _same(r[k], g[k]), (seed, k)


def test_bad_shape_rejected_without_device():
    import ctypes
    L = _lib.load()
    prm = _lib.SlmPreprocessParams(1.0, 0.95, -0.5, 0.0, 2, 1)
    rc = L.slm_preprocess(ctypes.c_void_p(16), 0, 1, 5, ctypes.byref(prm), ctypes.c_void_p(16), None, None, None,
                          None, None, None, None, None, None, None)
    assert rc == _lib.SLM_ERR_ARGS
    assert b"at least 2 pixels" in L.slm_last_error()


def test_numba_compiled_reference_functions(reference_dir):
    """The reference's njit functions compiled by numba (its production
    build) against the oracle: break_out_of_loop, check_has_loop (speed,
    divergence, curl), fix_blockages, and numba's double threshold compare.
    (find_and_fix_loops itself does not compile under current numba: its
    uint32 counter plus an int promotes to float64, which numba refuses as an
    index.)"""
    numba = pytest.importorskip("numba")
    import importlib.util
    import types
    dec = types.ModuleType("numba.decorators")
    dec.njit = numba.njit
    core = types.ModuleType("streamlines.core")
    core.Core = type("Core", (), {})
    pkg = types.ModuleType("streamlines")
    pkg.core = core
    saved = {k: sys.modules.get(k) for k in ("numba.decorators", "streamlines", "streamlines.core")}
    sys.modules.update({"numba.decorators": dec, "streamlines": pkg, "streamlines.core": core})
    try:
        spec = importlib.util.spec_from_file_location(
            "reference_preprocess_numba", os.path.join(reference_dir, "python", "streamlines", "preprocess.py"))
        mod = importlib.util.module_from_spec(spec)
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    rng = np.random.default_rng(1)
    nx, ny = 30, 25
    for _ in range(100):
        roi = rng.standard_normal((nx, ny)).astype(np.float32)
        roi[rng.random(roi.shape) < 0.05] = np.nan
        u = np.zeros((nx, ny), np.float32)
        v = np.zeros((nx, ny), np.float32)
        x, y = int(rng.integers(1, nx - 1)), int(rng.integers(1, ny - 1))
        mod.break_out_of_loop(np.array([x, y], np.uint32), u, v, roi, nx, ny)
        eu, ev = D.break_vector(roi, x, y)
        assert u[x, y].view(np.uint32) == eu.view(np.uint32) and v[x, y].view(np.uint32) == ev.view(np.uint32)
    u = rng.uniform(-1, 1, (2000, 2, 2)).astype(np.float32)
    v = rng.uniform(-1, 1, (2000, 2, 2)).astype(np.float32)
    got = np.array([mod.check_has_loop(0, 0, u[k], v[k]) for k in range(2000)], np.float32)
    uu = np.zeros((2, 2 * 2000), np.float32)
    vv = np.zeros((2, 2 * 2000), np.float32)
    for k in range(2000):  # cells (0, 2k) of a 2 x 4000 grid hold the samples
        uu[:, 2 * k:2 * k + 2] = u[k]
        vv[:, 2 * k:2 * k + 2] = v[k]
    for thr, col in ((0.5, 0), (0.0, 1)):
        cells = D.loop_cells(uu, vv, vecsum_threshold=2.0, divergence_threshold=10.0, curl_threshold=0.0)
        assert cells[0, ::2].all()
    # speed / divergence / curl, one by one, through the thresholds' strictness
    speed_ref, div_ref = got[:, 0], got[:, 1]
    for k in range(0, 2000, 97):
        for t, want in ((np.float64(speed_ref[k]), False), (np.nextafter(np.float64(speed_ref[k]), 9.0), True)):
            c = D.loop_cells(uu[:, 2 * k:2 * k + 2], vv[:, 2 * k:2 * k + 2], vecsum_threshold=t,
                             divergence_threshold=10.0, curl_threshold=0.0)
            assert bool(c[0, 0]) == want, (k, t)
        for t, want in ((np.float64(div_ref[k]), True), (np.nextafter(np.float64(div_ref[k]), -9.0), False)):
            c = D.loop_cells(uu[:, 2 * k:2 * k + 2], vv[:, 2 * k:2 * k + 2], vecsum_threshold=2.0,
                             divergence_threshold=t, curl_threshold=0.0)
            assert bool(c[0, 0]) == want, (k, t)

    @numba.njit
    def less(a, t):
        return a < t
    assert less(np.float32(0.95), 0.95)  # numba compares float32 with float64 in double
    codes = rng.choice(np.array([0, 1, 2, 4, 8, 16, 32, 64, 128, 3, 17, 96], np.uint8), (20, 20))
    nbr = rng.choice(np.array([0, 1, 2, 4, 8, 16, 32, 64, 128, 5, 24, 129], np.uint8), (20, 20))
    u = np.ones((20, 20), np.float32)
    v = np.ones((20, 20), np.float32)
    mod.fix_blockages(np.stack(np.where(codes)).T.astype(np.uint32), codes,
                      np.stack(np.where(nbr)).T.astype(np.uint32), nbr, u, v, False)
    eu = np.ones((20, 20), np.float32)
    ev = np.ones((20, 20), np.float32)
    for arr in (codes, nbr):
        xs, ys = np.nonzero(arr)
        dx, dy = D.flow_vectors(arr[xs, ys])
        eu[xs, ys] = np.where(dx != 0, dx.astype(np.float32) * D._INV_SQRT2_F32, np.float32(0.0))
        ev[xs, ys] = np.where(dy != 0, dy.astype(np.float32) * D._INV_SQRT2_F32, np.float32(0.0))
    assert np.array_equal(u.view(np.uint32), eu.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), ev.view(np.uint32))
