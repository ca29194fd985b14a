"""GPU KDE kernels against the oracle.

Histograms are integer counts: bit-exact.  Smoothed pdfs are fp64 sums of
the reference's terms in the reference's order, rounded to float; exp() and
cos() come from CUDA instead of the host libm, so the tolerance is stated per
point: relative error median <= 1e-7 and 99th percentile <= 1e-6 (max <= 1e-5),
relative to the pdf's maximum.
"""
import numpy as np
import pytest
import torch

import oracle as O
from kde_cases import bivariate, univariate
from slm_b200 import kde, kernels

pytestmark = pytest.mark.gpu
SHAPES = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]


def _close(got, want):
    scale = max(float(np.abs(want).max()), 1e-30)
    rel = np.abs(got.astype(np.float64) - want.astype(np.float64)) / scale
    assert np.median(rel) <= 1e-7, np.median(rel)
    assert np.percentile(rel, 99) <= 1e-6, np.percentile(rel, 99)
    assert rel.max() <= 1e-5, rel.max()


@pytest.mark.parametrize("kind", SHAPES)
@pytest.mark.parametrize("nb,npp", [(2048, 256), (8192, 1024)])
def test_univariate_kernels(kind, nb, npp):
    d, prm = univariate(kind, n_hist_bins=nb, n_pdf_points=npp, n=200000)
    data = np.ascontiguousarray(d.logx_data.reshape(-1), dtype=np.float32)
    hist_o = O.histogram_univariate(prm, data)
    pdf_o = O.pdf_univariate(prm, hist_o)
    data_d = torch.from_numpy(data).cuda()
    hist_d = torch.zeros(nb, dtype=torch.uint32, device="cuda")
    kernels.histogram_univariate(prm, data_d, hist_d)
    pdf_d = torch.zeros(npp, dtype=torch.float32, device="cuda")
    kernels.pdf_univariate(prm, hist_d, pdf_d)
    torch.cuda.synchronize()
    assert np.array_equal(hist_d.cpu().numpy(), hist_o)
    _close(pdf_d.cpu().numpy(), pdf_o)


@pytest.mark.parametrize("kind", SHAPES)
def test_bivariate_kernels(kind):
    d, prm = bivariate(kind, n=100000)
    nb, npp = int(d.n_hist_bins), int(d.n_pdf_points)
    data = np.ascontiguousarray(d.logxy_data, dtype=np.float32)
    hist_o = O.histogram_bivariate(prm, data)
    part_o = O.pdf_bivariate_rows(prm, hist_o)
    pdf_o = O.pdf_bivariate_cols(prm, part_o)
    data_d = torch.from_numpy(data).cuda()
    hist_d = torch.zeros(nb * nb, dtype=torch.uint32, device="cuda")
    kernels.histogram_bivariate(prm, data_d, hist_d)
    part_d = torch.zeros(nb * nb, dtype=torch.float32, device="cuda")
    kernels.pdf_bivariate_rows(prm, hist_d, part_d)
    pdf_d = torch.zeros(npp * npp, dtype=torch.float32, device="cuda")
    # the cols pass is checked on the oracle's partial pdf, the rows pass separately
    kernels.pdf_bivariate_cols(prm, torch.from_numpy(part_o).cuda(), pdf_d)
    torch.cuda.synchronize()
    assert np.array_equal(hist_d.cpu().numpy(), hist_o)
    _close(part_d.cpu().numpy(), part_o)
    _close(pdf_d.cpu().numpy(), pdf_o)


def test_estimate_univariate_pdf_end_to_end():
    d, prm = univariate("gaussian", n_hist_bins=8192, n_pdf_points=1024, n=300000)
    d.bandwidth = 2.0 / 2.0
    pdf, hist = kde.estimate_univariate_pdf(d)
    prm = kde.kde_params(d, "pdf_univariate")
    data = np.ascontiguousarray(d.logx_data.reshape(-1), dtype=np.float32)
    hist_o = O.histogram_univariate(prm, data).reshape(-1, 1)
    pdf_o = O.pdf_univariate(prm, hist_o).reshape(-1, 1)
    assert pdf.shape == (1024, 1) and hist.shape == (8192, 1)
    assert np.array_equal(hist, hist_o / (sum(hist_o) * d.bin_dx))
    _close(pdf, pdf_o / (sum(pdf_o) * d.bin_dx))


def test_estimate_bivariate_pdf_end_to_end():
    d, prm = bivariate("epanechnikov", n=50000)
    pdf, hist = kde.estimate_bivariate_pdf(d)
    assert pdf.shape == (64, 64) and hist.shape == (256, 256)
    assert abs(float(np.sum(hist) * d.bin_dx * d.bin_dy) - 1.0) < 1e-6
    assert abs(float(np.sum(pdf) * d.bin_dx * d.bin_dy) - 1.0) < 1e-4


def test_channel_threshold_from_device_pdf():
    """estimate_channel_threshold (device KDE + host consumers) equals the
    consumers run on the oracle's pdf of the same data."""
    from types import SimpleNamespace

    from slm_b200 import analysis as A
    rng = np.random.default_rng(21)
    nx, ny = 300, 280
    hill = rng.lognormal(2.5, 0.5, (nx, ny))
    chan = rng.lognormal(6.0, 0.8, (nx, ny))
    slt = np.where(rng.random((nx, ny)) < 0.08, chan, hill).astype(np.float32)
    sla = (slt * rng.uniform(0.5, 1.5, (nx, ny))).astype(np.float32)
    mask = rng.random((nx, ny)) < 0.05
    data = SimpleNamespace(slt_array=np.stack([slt, slt], 2), sla_array=np.stack([sla, sla], 2), mask_array=mask)
    d = A.compute_marginal_distribn_dslt(data)
    thr = A.estimate_channel_threshold(data)
    assert thr is not None and thr == d.channel_threshold_x
    # the same consumers on the oracle's pdf of the same selection
    prm = kde.kde_params(d, "pdf_univariate")
    x = np.ascontiguousarray(d.logx_data.reshape(-1), dtype=np.float32)
    hist_o = O.histogram_univariate(prm, x).reshape(-1, 1)
    pdf_o = O.pdf_univariate(prm, hist_o).reshape(-1, 1)
    pdf_o = pdf_o / (sum(pdf_o) * d.bin_dx)
    o = A.compute_marginal_distribn_dslt(data)  # fresh object, same data selection
    o.pdf = pdf_o.astype(np.float32)
    o.cdf = np.cumsum(o.pdf) * o.bin_dx
    o.pdf /= o.cdf[-1]
    o.cdf /= o.cdf[-1]
    for attr in ("mode_x", "channel_threshold_x"):
        if hasattr(o, attr):
            delattr(o, attr)
    o.find_modes()
    o.statistics()
    o.locate_threshold()
    assert o.mode_i == d.mode_i
    assert o.channel_threshold_i == d.channel_threshold_i
