"""The KDE consumers (modes, statistics, channel threshold, bivariate mode)
against the reference's own methods on identical pdfs (CPU only: the pdfs
are synthetic, as the device KDE would hand them over)."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

from slm_b200 import analysis as A


def _reference_analysis(reference_dir):
    stub = {"streamlines": types.ModuleType("streamlines"),
            "streamlines.kde": types.ModuleType("streamlines.kde"),
            "streamlines.core": types.ModuleType("streamlines.core"),
            "streamlines.useful": types.ModuleType("streamlines.useful")}
    stub["streamlines.core"].Core = type("Core", (), {})
    stub["streamlines.useful"].vprint = lambda *a, **k: None
    saved = {k: sys.modules.get(k) for k in stub}
    sys.modules.update(stub)
    try:
        path = os.path.join(reference_dir, "python", "streamlines", "analysis.py")
        spec = importlib.util.spec_from_file_location("reference_analysis", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


def _multimodal_pdf(logx_vec, seed, n_modes=3):
    rng = np.random.default_rng(seed)
    pdf = np.zeros_like(logx_vec)
    lo, hi = float(logx_vec.min()), float(logx_vec.max())
    for _ in range(n_modes):
        mu = rng.uniform(lo, hi)
        pdf += rng.uniform(0.2, 1.0) * np.exp(-0.5 * ((logx_vec - mu) / rng.uniform(0.1, 0.6)) ** 2)
    pdf += 0.01 * rng.random(pdf.shape)
    return pdf.astype(np.float32)


def _with_pdf(cls, data, pdf, **kw):
    d = cls(logx_array=data, logy_array=data, n_hist_bins=1024, n_pdf_points=pdf.shape[0], **kw)
    d.pdf = pdf.copy()
    d.cdf = np.cumsum(d.pdf) * d.bin_dx
    d.pdf /= d.cdf[-1]
    d.cdf /= d.cdf[-1]
    return d


@pytest.mark.parametrize("seed", range(12))
def test_univariate_consumers_match_reference(reference_dir, seed):
    R = _reference_analysis(reference_dir)
    rng = np.random.default_rng(100 + seed)
    data = np.log(rng.lognormal(3.0, 1.0, 5000)).astype(np.float32)
    kw = dict(search_cdf_min=[0.8, 0.95, 0.75][seed % 3], search_cdf_max=[0.999, 0.99, 0.9][seed % 3])
    probe = A.Univariate_distribution(logx_array=data, logy_array=data, n_hist_bins=1024, n_pdf_points=256)
    pdf = _multimodal_pdf(probe.logx_vec, seed)
    mine = _with_pdf(A.Univariate_distribution, data, pdf, **kw)
    ref = _with_pdf(R.Univariate_distribution, data, pdf, **kw)
    for d in (mine, ref):
        d.find_modes()
        d.statistics()
        d.locate_threshold()
    for k in ("mode_i", "mode_x", "mean", "stddev", "var", "raw_mean", "raw_stddev", "raw_var"):
        assert np.array_equal(np.asarray(getattr(mine, k)), np.asarray(getattr(ref, k))), k
    assert hasattr(mine, "channel_threshold_x") == hasattr(ref, "channel_threshold_x")
    if hasattr(ref, "channel_threshold_x"):
        assert mine.channel_threshold_i == ref.channel_threshold_i
        assert mine.channel_threshold_x == ref.channel_threshold_x


@pytest.mark.parametrize("seed", range(6))
def test_bivariate_mode_matches_reference(reference_dir, seed, monkeypatch):
    R = _reference_analysis(reference_dir)
    monkeypatch.setattr(np, "complex", complex, raising=False)  # the reference's np.complex (NumPy < 2)
    rng = np.random.default_rng(200 + seed)
    lx = np.log(rng.lognormal(2.0, 1.0, 4000)).astype(np.float32)
    ly = np.log(rng.lognormal(1.5, 0.8, 4000)).astype(np.float32)
    mine = A.Bivariate_distribution(logx_array=lx, logy_array=ly, n_hist_bins=512, n_pdf_points=64)
    ref = R.Bivariate_distribution(logx_array=lx, logy_array=ly, n_hist_bins=512, n_pdf_points=64)
    pdf = (_multimodal_pdf(mine.logx_mesh, seed) * _multimodal_pdf(mine.logy_mesh, seed + 50)).astype(np.float32)
    mine.pdf, ref.pdf = pdf.copy(), pdf.copy()
    mine.find_mode()
    ref.find_mode()
    assert mine.mode_ij == ref.mode_ij
    assert np.array_equal(mine.mode_xy, ref.mode_xy) and mine.mode_max == ref.mode_max


def test_threshold_search_floor_raises_like_reference():
    data = np.log(np.random.default_rng(1).lognormal(3.0, 1.0, 2000)).astype(np.float32)
    d = A.Univariate_distribution(logx_array=data, logy_array=data, n_hist_bins=512, n_pdf_points=128,
                                  search_cdf_min=0.5)
    d.pdf = _multimodal_pdf(d.logx_vec, 3)
    d.cdf = np.cumsum(d.pdf) / np.sum(d.pdf)
    d.find_modes()
    d.statistics()
    with pytest.raises(NameError):
        d.locate_threshold()


@pytest.mark.parametrize("estimate,expected", [(None, 150), (5000.0, 150), (4.0, 75.0), (220.0, 220.0)])
def test_subsegment_channel_threshold_clamps(monkeypatch, estimate, expected):
    """mapping.py:460-477: the guess when there is no estimate or it is above
    the maximum, half the guess below the minimum, else the estimate."""
    from types import SimpleNamespace

    from slm_b200 import mapping
    monkeypatch.setattr(A, "estimate_channel_threshold", lambda *a, **k: estimate)
    data = SimpleNamespace()
    assert mapping.subsegment_channel_threshold(data) == expected
    assert data.channel_threshold == expected
