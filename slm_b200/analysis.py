"""Distribution objects that drive the KDE stage.

``Univariate_distribution`` and ``Bivariate_distribution`` restate the
constructors and ``compute_kde_opencl`` methods of the reference's
``python/streamlines/analysis.py`` (:659-786 and :859-969): the data
selection, log-space ranges, bin and pdf spacings the KDE kernels read, the
gaussian bandwidth halving (:766-768) and the cdf normalisation.  The scipy
and sklearn alternatives, mode/threshold searches and plotting helpers of
those classes are not on the traced path and are not restated.
"""
from __future__ import annotations

import numpy as np

from . import kde

AVAILABLE_KERNELS = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]


class Univariate_distribution:
    def __init__(self, logx_array=None, logy_array=None, pixel_size=None, method="opencl",
                 n_hist_bins=2048, n_pdf_points=256, search_cdf_min=0.95, search_cdf_max=0.99,
                 logx_min=None, logy_min=None, logx_max=None, logy_max=None,
                 cl_src_path=None, cl_platform=None, cl_device=None, debug=False,
                 verbose=False, gpu_verbose=False):
        fmin = np.finfo(np.float32).min
        if logx_min is None:
            logx_min = logx_array[logx_array > fmin].min()
        if logx_max is None:
            logx_max = logx_array[logx_array > fmin].max()
        if logy_min is None:
            logy_min = logy_array[logy_array > fmin].min()
        if logy_max is None:
            logy_max = logy_array[logy_array > fmin].max()
        self.logx_data = logx_array[(logx_array >= logx_min) & (logx_array <= logx_max)
                                    & (logy_array >= logy_min) & (logy_array <= logy_max)]
        self.logx_data = self.logx_data.reshape((self.logx_data.shape[0], 1))
        self.logx_min = np.min(self.logx_data)
        self.logx_max = np.max(self.logx_data)
        self.logx_range = self.logx_max - self.logx_min
        self.logy_min = 0.0
        self.logy_max = 0.0
        self.logy_range = 0.0
        self.n_data = self.logx_data.shape[0]
        self.n_hist_bins = n_hist_bins
        self.n_pdf_points = n_pdf_points
        self.bin_dx = self.logx_range / self.n_hist_bins
        self.pdf_dx = self.logx_range / self.n_pdf_points
        self.bin_dy = 0.0
        self.pdf_dy = 0.0
        self.logx_vec = np.linspace(self.logx_min, self.logx_max,
                                    self.n_pdf_points).reshape((self.n_pdf_points, 1))
        self.logx_vec_histogram = np.linspace(self.logx_min, self.logx_max,
                                              self.n_hist_bins).reshape((self.n_hist_bins, 1))
        self.x_vec = np.exp(self.logx_vec)
        self.dlogx = self.logx_vec[1] - self.logx_vec[0]
        self.search_cdf_min = search_cdf_min
        self.search_cdf_max = search_cdf_max
        self.pixel_size = pixel_size
        self.cl_src_path = cl_src_path
        self.cl_platform = cl_platform
        self.cl_device = cl_device
        self.debug = debug
        self.verbose = verbose
        self.gpu_verbose = gpu_verbose

    def compute_kde_opencl(self, kernel="epanechnikov", bandwidth=0.15):
        """Histogram + kernel smoothing on the device (analysis.py:763-786)."""
        self.kernel = kernel
        self.bandwidth = bandwidth
        if self.kernel == "gaussian":
            self.bandwidth /= 2.0
        if self.kernel not in AVAILABLE_KERNELS:
            raise ValueError('PDF kernel "{}" is not among those available: {}'
                             .format(self.kernel, AVAILABLE_KERNELS))
        self.pdf, self.histogram = kde.estimate_univariate_pdf(self)
        self.cdf = np.cumsum(self.pdf) * self.bin_dx
        cdf_max = self.cdf[-1]
        self.pdf /= cdf_max
        self.cdf /= cdf_max


class Bivariate_distribution:
    def __init__(self, logx_array=None, logy_array=None, mask_array=None, pixel_size=None,
                 method="opencl", n_hist_bins=2048, n_pdf_points=256, logx_min=None,
                 logy_min=None, logx_max=None, logy_max=None, cl_src_path=None,
                 cl_platform=None, cl_device=None, debug=False, verbose=False,
                 gpu_verbose=False):
        self.logx_data = logx_array
        self.logy_data = logy_array
        fmin = np.finfo(np.float32).min
        if logx_min is None:
            logx_min = logx_array[logx_array > fmin].min()
        if logx_max is None:
            logx_max = logx_array[logx_array > fmin].max()
        if logy_min is None:
            logy_min = logy_array[logy_array > fmin].min()
        if logy_max is None:
            logy_max = logy_array[logy_array > fmin].max()
        sel = ((logx_array >= logx_min) & (logx_array <= logx_max)
               & (logy_array >= logy_min) & (logy_array <= logy_max))
        if mask_array is not None:
            sel = sel & (~mask_array)
        logxy_data = np.vstack([logx_array[sel], logy_array[sel]]).T
        self.logxy_data = logxy_data.copy().astype(dtype=np.float32)
        self.logx_mesh, self.logy_mesh = np.mgrid[logx_min:logx_max:complex(n_pdf_points),
                                                  logy_min:logy_max:complex(n_pdf_points)]
        self.logx_min = logx_min
        self.logx_max = logx_max
        self.logy_min = logy_min
        self.logy_max = logy_max
        self.logx_range = self.logx_max - self.logx_min
        self.logy_range = self.logy_max - self.logy_min
        self.n_data = self.logxy_data.shape[0]
        self.n_hist_bins = n_hist_bins
        self.n_pdf_points = n_pdf_points
        self.bin_dx = self.logx_range / self.n_hist_bins
        self.pdf_dx = self.logx_range / self.n_pdf_points
        self.bin_dy = self.logy_range / self.n_hist_bins
        self.pdf_dy = self.logy_range / self.n_pdf_points
        self.x_mesh = np.exp(self.logx_mesh)
        self.y_mesh = np.exp(self.logy_mesh)
        self.pixel_size = pixel_size
        self.cl_src_path = cl_src_path
        self.cl_platform = cl_platform
        self.cl_device = cl_device
        self.debug = debug
        self.verbose = verbose
        self.gpu_verbose = gpu_verbose

    def compute_kde_opencl(self, kernel="epanechnikov", bandwidth=0.10):
        """Histogram + separable smoothing on the device (analysis.py:955-969)."""
        self.kernel = kernel
        self.bandwidth = bandwidth
        if self.kernel not in AVAILABLE_KERNELS:
            raise ValueError('PDF kernel "{}" is not among those available: {}'
                             .format(self.kernel, AVAILABLE_KERNELS))
        self.pdf, self.histogram = kde.estimate_bivariate_pdf(self)
        self.cdf = np.cumsum(self.pdf) * self.bin_dx
