"""slm_preprocess on the GPU against the reference's golden vectors and the
oracle (bit-exact; the slope, an arctangent, within float32 rounding)."""
import glob
import os

import numpy as np
import pytest

import dtm_preprocess as D

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EXACT = ("uv_array", "uv_mask_array", "blockages_array", "blocked_neighbors_array", "where_looped_array",
         "roi_gradx_array", "roi_grady_array")


def _same(a, b):
    """Bit-exact, except that a NaN matches any NaN (the device's NaN bit
    pattern differs from the host's)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype == bool:
        return np.array_equal(a, b)
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        if not np.array_equal(na, nb):
            return False
        a, b = np.where(na, 0, a), np.where(nb, 0, b)
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _slope_close(a, b):
    # float32 arctangent (NumPy's vs the device's) times 180/pi: a few ulp
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)


def _gpu(roi, pixel_size, pad, normalize=True, **kw):
    from slm_b200.preprocess import conditioned_gradient_vector_field
    return conditioned_gradient_vector_field(roi, pixel_size, pad, do_normalize_speed=normalize, **kw)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "preprocess_*.npz"))))
def test_preprocess_matches_reference_golden(path):
    g = np.load(path)
    r = _gpu(g["roi"], float(g["pixel_size"]), int(g["pad_width"]), bool(g["do_normalize_speed"]))
    for k in EXACT:
        assert _same(getattr(r, k), g[k]), k
    assert r.n_loops == int(g["n_loops"])
    _slope_close(r.slope_array, g["slope_array"])


def _roi(nx, ny, seed, noise=0.3, dtype=np.float32, holes=0.0, plateaus=False):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)[:, None]
    y = np.arange(ny)[None, :]
    roi = 100.0 + 0.3 * x - 0.2 * y + 4.0 * np.sin(x / 9.0) * np.cos(y / 13.0) + noise * rng.standard_normal((nx, ny))
    if plateaus:
        roi = np.round(roi)
    roi = roi.astype(dtype)
    if holes:
        roi[rng.random((nx, ny)) < holes] = np.nan
    return roi


CASES = [
    dict(nx=2, ny=2, seed=1), dict(nx=2, ny=77, seed=2), dict(nx=9, ny=33, seed=3), dict(nx=33, ny=9, seed=4),
    dict(nx=300, ny=257, seed=5, holes=0.01), dict(nx=129, ny=200, seed=6, dtype=np.float64, plateaus=True),
    dict(nx=250, ny=250, seed=7, pixel_size=0.3, pad=0), dict(nx=64, ny=96, seed=8, pad=7, normalize=False),
    dict(nx=511, ny=513, seed=9, noise=0.05, pixel_size=2.0, holes=0.002),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "{}x{}".format(c["nx"], c["ny"]))
def test_preprocess_matches_oracle(case):
    c = dict(case)
    pixel_size, pad, normalize = c.pop("pixel_size", 1.0), c.pop("pad", 2), c.pop("normalize", True)
    roi = _roi(**c)
    o = D.conditioned_uv(roi, pixel_size, pad, do_normalize_speed=normalize)
    r = _gpu(roi, pixel_size, pad, normalize)
    for k in EXACT:
        assert _same(getattr(r, k), o[k]), k
    _slope_close(r.slope_array, o["slope_array"])
    # the combined mask: pad frame, NaN ROI pixels, NaN vectors
    frame = np.ones(r.mask_array.shape, bool)
    nx, ny = roi.shape
    frame[pad:pad + nx, pad:pad + ny] = np.isnan(roi)
    assert np.array_equal(r.mask_array, frame | o["uv_mask_array"])


def test_preprocess_thresholds_and_no_loops():
    roi = _roi(100, 120, 11, noise=0.5)
    a = _gpu(roi, 1.0, 2, vecsum_threshold=0.0)  # speed < 0 never holds: no loops
    assert a.n_loops == 0
    o = D.conditioned_uv(roi, 1.0, 2, vecsum_threshold=0.0)
    assert _same(a.uv_array, o["uv_array"])
    b = _gpu(roi, 1.0, 2, divergence_threshold=0.25, curl_threshold=0.1)
    o = D.conditioned_uv(roi, 1.0, 2, divergence_threshold=0.25, curl_threshold=0.1)
    assert b.n_loops == o["n_loops"] > 0
    assert _same(b.uv_array, o["uv_array"])


def test_preprocess_device_resident_feeds_the_tracer():
    """download=False keeps uv and mask on the device in the tracer's layout."""
    import torch
    roi = _roi(80, 70, 12)
    r = _gpu(roi, 1.0, 2, download=False)
    h = _gpu(roi, 1.0, 2)
    assert r.uv_array.is_cuda and tuple(r.uv_array.shape) == (84, 74, 2)
    assert torch.equal(r.uv_array.cpu(), torch.from_numpy(h.uv_array))
    assert 4 * int(r.n_loop_cells.item()) == h.n_loops


def test_preprocess_class_mirrors_reference():
    from types import SimpleNamespace

    from slm_b200.preprocess import Preprocess
    roi = _roi(60, 50, 13, holes=0.02)
    masks = []
    state = SimpleNamespace(do_condition=True, add_active_mask=masks.append)
    geodata = SimpleNamespace(roi_array=roi, pixel_size=1.0, pad_width=2)
    p = Preprocess(state, {"preprocess": {"do_normalize_speed": True, "vecsum_threshold": 0.95,
                                          "divergence_threshold": -0.5, "curl_threshold": 0.0}}, geodata)
    p.do()
    o = D.conditioned_uv(roi, 1.0, 2)
    assert _same(p.uv_array, o["uv_array"])
    assert np.array_equal(masks[0]["uv"], o["uv_mask_array"])
    assert p.n_loops == o["n_loops"]
    assert p.where_blockages_array.shape[1] == 2
    state.do_condition = False
    with pytest.raises(NameError):
        Preprocess(state, {}, geodata).do()


def test_preprocess_full_size_properties():
    """2048^2: unit vectors wherever the field is defined, identical to the
    oracle on a band of rows, repeatable run to run."""
    from slm_b200 import synth
    dtm = synth.incised_dtm(2048, 3, 400).astype(np.float32)
    r1 = _gpu(dtm, 2.0, 2, download=False)
    r2 = _gpu(dtm, 2.0, 2, download=False)
    import torch
    assert torch.equal(r1.uv_array, r2.uv_array)
    uv = r1.uv_array.double()
    n = torch.sqrt((uv ** 2).sum(-1))
    ok = r1.uv_mask_array == 0
    assert torch.all((torch.abs(n[ok] - 1.0) < 1e-6) | (n[ok] == 0.0))  # flat pixels stay (0, 0)
    band = dtm[1000:1064]
    o = D.conditioned_uv(band, 2.0, 2)
    # rows 2..61 of the band see the same 5-row neighbourhood as in the full grid
    full = r1.uv_array[1000 + 2 + 2:1000 + 62 + 2, 2:-2].cpu().numpy()
    part = o["uv_array"][2 + 2:62 + 2, 2:-2]
    assert _same(full, part)
