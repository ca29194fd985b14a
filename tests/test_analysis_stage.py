"""The Analysis stage mirror against the reference's own Analysis class (CPU).

Both run with the same deterministic CPU stand-in for the KDE (the pdfs the
device would hand over), so what is compared is the stage's own logic: which
fields and directions each marginal and joint pdf takes, the log limits,
the data selection, and the modes, statistics and thresholds found."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

from slm_b200 import analysis as A
from test_analysis_consumers import _reference_analysis


def fake_univariate(d, do_detrend=False, logx_vec=None):
    h, _ = np.histogram(d.logx_data.ravel(), bins=d.n_hist_bins, range=(d.logx_min, d.logx_max))
    hist = h.astype(np.float64).reshape(-1, 1)
    k = d.n_hist_bins // d.n_pdf_points
    pdf = np.convolve(h.reshape(-1, k).sum(1).astype(np.float64), np.ones(5) / 5, "same").reshape(-1, 1)
    return pdf / (np.sum(pdf) * d.bin_dx), hist / (np.sum(hist) * d.bin_dx)


def fake_bivariate(d):
    x, y = d.logxy_data[:, 0], d.logxy_data[:, 1]
    h, _, _ = np.histogram2d(x, y, bins=d.n_hist_bins, range=((d.logx_min, d.logx_max), (d.logy_min, d.logy_max)))
    k = d.n_hist_bins // d.n_pdf_points
    pdf = h.reshape(d.n_pdf_points, k, d.n_pdf_points, k).sum((1, 3))
    return pdf / (np.sum(pdf) * d.bin_dx * d.bin_dy), h / (np.sum(h) * d.bin_dx * d.bin_dy)


def _fields(seed):
    rng = np.random.default_rng(seed)
    nxp, nyp = 90, 80
    hill = rng.lognormal(2.5, 0.5, (nxp, nyp, 2))
    chan = rng.lognormal(6.0, 0.8, (nxp, nyp, 2))
    slt = np.where(rng.random((nxp, nyp, 1)) < 0.08, chan, hill).astype(np.float32)
    sla = (slt * rng.uniform(0.5, 1.5, slt.shape)).astype(np.float32)
    slc = (slt * rng.uniform(0.2, 3.0, slt.shape)).astype(np.float64)
    mask = rng.random((nxp, nyp)) < 0.05
    return types.SimpleNamespace(slt_array=slt, sla_array=sla, slc_array=slc, mask_array=mask)


def _params():
    p = dict(A.ANALYSIS_PARAMETERS)
    p.update(n_hist_bins=1024, n_pdf_points=128)
    for k in list(p):
        if k.startswith("do_marginal") or k.startswith("do_joint"):
            p[k] = True
    p["do_marginal_distbn_usla"] = False  # raises without data in the reference (tested below)
    return {"analysis": p}


@pytest.mark.parametrize("seed", [0, 1])
def test_analysis_stage_matches_reference(reference_dir, seed, monkeypatch):
    R = _reference_analysis(reference_dir)
    monkeypatch.setattr(np, "complex", complex, raising=False)  # the reference's np.complex (NumPy < 2)
    monkeypatch.setattr(A.kde, "estimate_univariate_pdf", fake_univariate)
    monkeypatch.setattr(A.kde, "estimate_bivariate_pdf", fake_bivariate)
    R.kde.estimate_univariate_pdf = fake_univariate
    R.kde.estimate_bivariate_pdf = fake_bivariate
    data = _fields(seed)
    state = types.SimpleNamespace(verbose=False, gpu_verbose=False, debug=False, cl_src_path=None,
                                  cl_platform=0, cl_device=0)
    geodata = types.SimpleNamespace(roi_pixel_size=2.0)
    params = _params()

    class RefCore:
        def __init__(self, st, imported):  # Core sets the section's keys and the verbosity
            for k, v in imported["analysis"].items():
                setattr(self, k, v)
            self.verbose = False

        def print(self, *a, **k):
            pass
    ref = R.Analysis.__new__(R.Analysis)
    RefCore.__init__(ref, state, params)
    ref.__dict__.update(state=state, geodata=geodata, preprocess=None, trace=data, mapping=None,
                        print=lambda *a, **k: None)
    mine = A.Analysis(state, params, geodata, None, data)
    ref.do()
    mine.do()
    with pytest.raises(AttributeError):
        ref.compute_marginal_distribn_usla()
    with pytest.raises(AttributeError):
        mine.compute_marginal_distribn_usla()
    ref.compute_marginal_distribn_usla(data)
    mine.compute_marginal_distribn_usla(data)
    for name, *_ in A.MARGINALS:
        a, b = getattr(mine, "mpdf_" + name), getattr(ref, "mpdf_" + name)
        for k in ("mode_i", "mode_x", "mean", "stddev", "raw_mean", "n_data", "logx_min", "logx_max"):
            assert np.array_equal(np.asarray(getattr(a, k)), np.asarray(getattr(b, k))), (name, k)
        assert np.array_equal(a.pdf, b.pdf), name
        assert getattr(a, "channel_threshold_x", None) == getattr(b, "channel_threshold_x", None), name
    for name, *_ in A.JOINTS:
        a, b = getattr(mine, "jpdf_" + name), getattr(ref, "jpdf_" + name)
        assert a.mode_ij == b.mode_ij and np.array_equal(a.mode_xy, b.mode_xy), name
        assert np.array_equal(a.logxy_data, b.logxy_data), name
    # the channel threshold of a data object, as the mapping pass asks for it
    assert mine.estimate_channel_threshold(data) == ref.estimate_channel_threshold(data)
