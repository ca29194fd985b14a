"""Seeded KDE inputs shared by the CPU and GPU KDE tests."""
import numpy as np

from slm_b200.analysis import Bivariate_distribution, Univariate_distribution
from slm_b200.kde import kde_params, prepare_bivariate, prepare_univariate


def univariate(kind="gaussian", n=20000, n_hist_bins=2048, n_pdf_points=256, bandwidth=2.0, seed=1):
    rng = np.random.default_rng(seed)
    x = np.log(rng.lognormal(3.0, 0.8, size=n)).astype(np.float32)
    d = Univariate_distribution(logx_array=x, logy_array=x, n_hist_bins=n_hist_bins,
                                n_pdf_points=n_pdf_points, cl_device=0)
    d.kernel, d.bandwidth = kind, bandwidth / 2.0 if kind == "gaussian" else bandwidth
    prepare_univariate(d)
    return d, kde_params(d, "pdf_univariate")


def bivariate(kind="gaussian", n=20000, n_hist_bins=256, n_pdf_points=64, bandwidth=5.0, seed=2):
    rng = np.random.default_rng(seed)
    x = np.log(rng.lognormal(2.0, 0.6, size=n)).astype(np.float32)
    y = (0.5 * x + np.log(rng.lognormal(1.0, 0.4, size=n))).astype(np.float32)
    d = Bivariate_distribution(logx_array=x, logy_array=y, n_hist_bins=n_hist_bins,
                               n_pdf_points=n_pdf_points, cl_device=0)
    d.kernel, d.bandwidth = kind, bandwidth
    prepare_bivariate(d)
    return d, kde_params(d, "pdf_bivariate_rows")
