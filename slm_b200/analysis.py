"""Distribution objects that drive the KDE stage, and their consumers.

``Univariate_distribution`` and ``Bivariate_distribution`` restate the
constructors and ``compute_kde_opencl`` methods of the reference's
``python/streamlines/analysis.py`` (:659-786 and :859-969): the data
selection, log-space ranges, bin and pdf spacings the KDE kernels read, the
gaussian bandwidth halving (:766-768) and the cdf normalisation.  The
consumers of the device pdfs follow: the univariate ``statistics``,
``find_modes`` and ``locate_threshold`` (:788-853), the bivariate
``find_mode`` (:971-984), and ``compute_marginal_distribn`` /
``estimate_channel_threshold`` (Analysis, :120-188, :236-256), which give
the mapping stage its channel threshold from the pdf of the downstream slt.
The scipy and sklearn KDE alternatives and the plotting helpers are not
restated.
"""
from __future__ import annotations

import numpy as np
from scipy.signal import argrelextrema
from scipy.stats import norm

from . import kde
from .useful import vprint

AVAILABLE_KERNELS = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]


def _data_limits(a, lo, hi):
    """The log-space limits of ``a`` where not given: its extremes above
    float32's lowest value (the "no data" marker of the log arrays)."""
    if lo is None or hi is None:
        valid = a[a > np.finfo(np.float32).min]
        lo = valid.min() if lo is None else lo
        hi = valid.max() if hi is None else hi
    return lo, hi


def _set_in_order(obj, table):
    """Evaluate a (name, derivation) attribute table on ``obj`` in order."""
    for name, derive in table:
        setattr(obj, name, derive(obj))


# What the KDE stage and its consumers read from a univariate distribution,
# and how each value follows from the selected data (the reference's
# analysis.py:665-717 derives the same values).  Evaluated in order on the
# object; ``logx_data`` (the selected log data, one column) is set first.
#   read by the histogram / pdf kernels (kde.estimate_univariate_pdf):
#     logx_data, n_data, logx_min, logx_range, n_hist_bins, n_pdf_points,
#     bin_dx, pdf_dx, and the unused y axis (zeros) of the shared parameter set
#   read by the consumers (cdf, statistics, find_modes, locate_threshold):
#     logx_vec, x_vec, bin_dx, search_cdf_min / max
_UNIVARIATE_TABLE = (
    ("logx_min", lambda d: np.min(d.logx_data)),          # the data's, not the selection limits
    ("logx_max", lambda d: np.max(d.logx_data)),
    ("logx_range", lambda d: d.logx_max - d.logx_min),
    ("logy_min", lambda d: 0.0),
    ("logy_max", lambda d: 0.0),
    ("logy_range", lambda d: 0.0),
    ("n_data", lambda d: d.logx_data.shape[0]),
    ("bin_dx", lambda d: d.logx_range / d.n_hist_bins),
    ("pdf_dx", lambda d: d.logx_range / d.n_pdf_points),
    ("bin_dy", lambda d: 0.0),
    ("pdf_dy", lambda d: 0.0),
    ("logx_vec", lambda d: np.linspace(d.logx_min, d.logx_max, d.n_pdf_points).reshape((d.n_pdf_points, 1))),
    ("logx_vec_histogram", lambda d: np.linspace(d.logx_min, d.logx_max,
                                                 d.n_hist_bins).reshape((d.n_hist_bins, 1))),
    ("x_vec", lambda d: np.exp(d.logx_vec)),
    ("dlogx", lambda d: d.logx_vec[1] - d.logx_vec[0]),
)

# The same for a bivariate distribution (the reference's analysis.py:
# 859-900).  ``logxy_data`` (float32 rows of the selected (x, y) pairs) and
# the four limits (given, or the data's extremes) are set first.
#   read by the histogram / rows / cols kernels (kde.estimate_bivariate_pdf):
#     logxy_data, n_data, logx_min, logy_min, the ranges, n_hist_bins,
#     n_pdf_points, bin_dx / bin_dy, pdf_dx / pdf_dy
#   read by the consumers (cdf, find_mode): bin_dx, x_mesh, y_mesh
_BIVARIATE_TABLE = (
    ("logx_range", lambda d: d.logx_max - d.logx_min),
    ("logy_range", lambda d: d.logy_max - d.logy_min),
    ("n_data", lambda d: d.logxy_data.shape[0]),
    ("bin_dx", lambda d: d.logx_range / d.n_hist_bins),
    ("pdf_dx", lambda d: d.logx_range / d.n_pdf_points),
    ("bin_dy", lambda d: d.logy_range / d.n_hist_bins),
    ("pdf_dy", lambda d: d.logy_range / d.n_pdf_points),
    ("x_mesh", lambda d: np.exp(d.logx_mesh)),
    ("y_mesh", lambda d: np.exp(d.logy_mesh)),
)

# constructor arguments kept as attributes unchanged
_PASSED_THROUGH = ("pixel_size", "cl_src_path", "cl_platform", "cl_device", "debug", "verbose", "gpu_verbose")


class Univariate_distribution:
    """Log-space data of one quantity and the KDE of it (the reference's
    streamlines.analysis.Univariate_distribution, OpenCL method).  The
    selection keeps the x values whose (x, y) pair lies inside the limits;
    the derived attributes follow ``_UNIVARIATE_TABLE``."""

    def __init__(self, logx_array=None, logy_array=None, pixel_size=None, method="opencl",
                 n_hist_bins=2048, n_pdf_points=256, search_cdf_min=0.95, search_cdf_max=0.99,
                 logx_min=None, logy_min=None, logx_max=None, logy_max=None,
                 cl_src_path=None, cl_platform=None, cl_device=None, debug=False,
                 verbose=False, gpu_verbose=False):
        x_lo, x_hi = _data_limits(logx_array, logx_min, logx_max)
        y_lo, y_hi = _data_limits(logy_array, logy_min, logy_max)
        inside = (logx_array >= x_lo) & (logx_array <= x_hi) & (logy_array >= y_lo) & (logy_array <= y_hi)
        self.logx_data = logx_array[inside].reshape((-1, 1))
        self.n_hist_bins, self.n_pdf_points = n_hist_bins, n_pdf_points
        self.search_cdf_min, self.search_cdf_max = search_cdf_min, search_cdf_max
        _set_in_order(self, _UNIVARIATE_TABLE)
        args = locals()
        for name in _PASSED_THROUGH:
            setattr(self, name, args[name])

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

    def statistics(self):
        """pdf-weighted mean and spread in log space, and of the raw data
        (analysis.py:788-798); stored exponentiated."""
        w = self.pdf
        total = np.sum(w)
        mu = np.sum(self.logx_vec * w) / total
        var = np.sum((self.logx_vec - mu) ** 2 * w) / total
        self.mean, self.stddev, self.var = np.exp(mu), np.exp(np.sqrt(var)), np.exp(var)
        self.raw_mean = np.exp(self.logx_data.mean())
        self.raw_stddev = np.exp(self.logx_data.std())
        self.raw_var = np.exp(self.logx_data.var())

    def find_modes(self):
        """The first local maximum (3 points either side) at or above half the
        global maximum's x (analysis.py:800-812); the middle point and 100 m
        when there is none."""
        flat = np.reshape(self.pdf, self.pdf.shape[0])
        approx_mode = np.round(self.x_vec[self.pdf == self.pdf.max()][0], 2)
        peaks = [i for i in argrelextrema(flat, np.greater, order=3)[0]
                 if self.x_vec[i] >= approx_mode * 0.5]
        if peaks:
            self.mode_i = peaks[0]
            self.mode_x = self.x_vec[peaks[0]][0]
        else:
            self.mode_i = self.pdf.shape[0] // 2
            self.mode_x = 100.0

    def locate_threshold(self):
        """Channel threshold: the first local minimum (3 points either side,
        plus the last point) of the pdf divided by the log-normal of its own
        statistics, at or beyond the mode, whose cdf lies in
        [search_cdf_min, search_cdf_max]; search_cdf_min is lowered by 0.01
        down to 0.70 until one qualifies (analysis.py:814-853).  Needs
        find_modes and statistics first."""
        n = self.pdf.shape[0]
        log_normal = norm.pdf(np.log(self.x_vec), np.log(self.mean), np.log(self.stddev))
        ratio = np.reshape(self.pdf / log_normal, n)
        minima = np.concatenate((argrelextrema(ratio, np.less, order=3)[0], np.array([n - 1])))
        lo = self.search_cdf_min
        if lo < 0.70:  # the reference's loop never binds its result list
            raise NameError("name 'extrema_i' is not defined")
        chosen = []
        while lo >= 0.70:
            chosen = [i for i in minima if self.x_vec[i] >= self.mode_x
                      and self.cdf[i] >= lo and self.cdf[i] <= self.search_cdf_max]
            if chosen:
                break
            lo -= 0.01
        if chosen:
            self.channel_threshold_i = chosen[0]
            self.channel_threshold_x = self.x_vec[chosen[0]][0]


class Bivariate_distribution:
    """Log-space (x, y) pairs and their 2-D KDE (the reference's
    streamlines.analysis.Bivariate_distribution, OpenCL method).  The
    selection keeps the pairs inside the limits (and outside ``mask_array``);
    the pdf mesh spans the limits; the derived attributes follow
    ``_BIVARIATE_TABLE``."""

    def __init__(self, logx_array=None, logy_array=None, mask_array=None, pixel_size=None,
                 method="opencl", n_hist_bins=2048, n_pdf_points=256, logx_min=None,
                 logy_min=None, logx_max=None, logy_max=None, cl_src_path=None,
                 cl_platform=None, cl_device=None, debug=False, verbose=False,
                 gpu_verbose=False):
        self.logx_data, self.logy_data = logx_array, logy_array
        self.logx_min, self.logx_max = _data_limits(logx_array, logx_min, logx_max)
        self.logy_min, self.logy_max = _data_limits(logy_array, logy_min, logy_max)
        inside = ((logx_array >= self.logx_min) & (logx_array <= self.logx_max)
                  & (logy_array >= self.logy_min) & (logy_array <= self.logy_max))
        if mask_array is not None:
            inside &= ~mask_array
        self.logxy_data = np.stack([logx_array[inside], logy_array[inside]], axis=1).astype(np.float32)
        n = complex(n_pdf_points)
        self.logx_mesh, self.logy_mesh = np.mgrid[self.logx_min:self.logx_max:n, self.logy_min:self.logy_max:n]
        self.n_hist_bins, self.n_pdf_points = n_hist_bins, n_pdf_points
        _set_in_order(self, _BIVARIATE_TABLE)
        args = locals()
        for name in _PASSED_THROUGH:
            setattr(self, name, args[name])

    def compute_kde_opencl(self, kernel="epanechnikov", bandwidth=0.10):
        """Histogram + separable smoothing on the device (analysis.py:955-969)."""
        self.kernel = kernel
        self.bandwidth = bandwidth
        if self.kernel not in AVAILABLE_KERNELS:
            raise ValueError('PDF kernel "{}" is not among those available: {}'
                             .format(self.kernel, AVAILABLE_KERNELS))
        self.pdf, self.histogram = kde.estimate_bivariate_pdf(self)
        self.cdf = np.cumsum(self.pdf) * self.bin_dx

    def find_mode(self):
        """(x, y) of the pdf maximum, ignoring x or y <= 3 (analysis.py:971-984)."""
        f = self.pdf.copy()
        f[(self.x_mesh <= 3.0) | (self.y_mesh <= 3.0)] = 0.0
        ij = np.unravel_index(np.argmax(f, axis=None), f.shape)
        self.mode_max = f[ij[0], ij[1]]
        self.mode_ij = ij
        self.mode_xy = np.array([self.x_mesh[ij[0], 0], self.y_mesh[0, ij[1]]])


ANALYSIS_DEFAULTS = {"n_hist_bins": 2048, "n_pdf_points": 256, "search_cdf_min": 0.8, "search_cdf_max": 0.999,
                     "marginal_distbn_kde_kernel": "epanechnikov", "marginal_distbn_kde_bandwidth": 10.0,
                     "pdf_slt_min": 1, "pdf_sla_min": 1}


def compute_marginal_distribn(x_array, y_array, mask_array=None, up_down_idx_x=0, up_down_idx_y=0,
                              n_hist_bins=2048, n_pdf_points=256, kernel="epanechnikov", bandwidth=10.0,
                              logx_min=None, logy_min=None, logx_max=None, logy_max=None,
                              search_cdf_min=0.8, search_cdf_max=0.999, pixel_size=None, cl_platform=0,
                              cl_device=0, verbose=False):
    """Analysis.compute_marginal_distribn with the device KDE (analysis.py:136-188):
    the positive (x, y) pairs of the unmasked pixels in log space, the pdf,
    then find_modes, statistics and locate_threshold."""
    if mask_array is not None:
        tx = x_array[~mask_array, up_down_idx_x].astype(np.float32)
        ty = y_array[~mask_array, up_down_idx_y].astype(np.float32)
    else:
        tx = x_array[:, :, up_down_idx_x].astype(np.float32).ravel()
        ty = y_array[:, :, up_down_idx_y].astype(np.float32).ravel()
    keep = (tx > 0.0) & (ty > 0.0)
    d = Univariate_distribution(logx_array=np.log(tx[keep]), logy_array=np.log(ty[keep]), pixel_size=pixel_size,
                                n_hist_bins=n_hist_bins, n_pdf_points=n_pdf_points, logx_min=logx_min,
                                logy_min=logy_min, logx_max=logx_max, logy_max=logy_max,
                                search_cdf_min=search_cdf_min, search_cdf_max=search_cdf_max,
                                cl_platform=cl_platform, cl_device=cl_device, verbose=verbose)
    d.compute_kde_opencl(kernel=kernel, bandwidth=bandwidth)
    d.find_modes()
    d.statistics()
    d.locate_threshold()
    return d


def estimate_channel_threshold(data, params=None, pixel_size=None):
    """Analysis.estimate_channel_threshold (analysis.py:120-134): the
    threshold located on the marginal pdf of the downstream slt, or None when
    none qualifies.  ``params``: the 'analysis' section of the job's
    parameters (defaults: json/defaults.json)."""
    return getattr(compute_marginal_distribn_dslt(data, params, pixel_size), "channel_threshold_x", None)


def compute_marginal_distribn_dslt(data, params=None, pixel_size=None):
    """Analysis.compute_marginal_distribn_dslt (analysis.py:236-256): the
    downstream slt limited by sla, pdf_slt_min / pdf_sla_min as log limits."""
    p = dict(ANALYSIS_DEFAULTS)
    p.update(params or {})
    lim = lambda k: np.log(p[k]) if k in p and p[k] is not None else None  # noqa: E731
    d = compute_marginal_distribn(data.slt_array, data.sla_array, data.mask_array, 0, 0,
                                  n_hist_bins=p["n_hist_bins"], n_pdf_points=p["n_pdf_points"],
                                  kernel=p["marginal_distbn_kde_kernel"],
                                  bandwidth=p["marginal_distbn_kde_bandwidth"],
                                  logx_min=lim("pdf_slt_min"), logx_max=lim("pdf_slt_max"),
                                  logy_min=lim("pdf_sla_min"), logy_max=lim("pdf_sla_max"),
                                  search_cdf_min=p["search_cdf_min"], search_cdf_max=p["search_cdf_max"],
                                  pixel_size=pixel_size)
    return d


def compute_joint_distribn(x_array, y_array, mask_array=None, up_down_idx_x=0, up_down_idx_y=0, n_hist_bins=2048,
                           n_pdf_points=256, kernel="gaussian", bandwidth=5.0, logx_min=None, logy_min=None,
                           logx_max=None, logy_max=None, pixel_size=None, cl_platform=0, cl_device=0,
                           verbose=False):
    """Analysis.compute_joint_distribn with the device KDE (analysis.py:326-381):
    the positive (x, y) pairs of the unmasked pixels in log space, the
    bivariate pdf, then find_mode."""
    if mask_array is not None:
        tx = x_array[~mask_array, up_down_idx_x].copy().astype(np.float32)
        ty = y_array[~mask_array, up_down_idx_y].copy().astype(np.float32)
    else:
        tx = x_array[:, :, up_down_idx_x].copy().ravel().astype(np.float32)
        ty = y_array[:, :, up_down_idx_y].copy().ravel().astype(np.float32)
    keep = (tx > 0.0) & (ty > 0.0)
    d = Bivariate_distribution(logx_array=np.log(tx[keep]), logy_array=np.log(ty[keep]), pixel_size=pixel_size,
                               n_hist_bins=n_hist_bins, n_pdf_points=n_pdf_points, logx_min=logx_min,
                               logy_min=logy_min, logx_max=logx_max, logy_max=logy_max,
                               cl_platform=cl_platform, cl_device=cl_device, verbose=verbose)
    d.compute_kde_opencl(kernel=kernel, bandwidth=bandwidth)
    d.find_mode()
    return d


ANALYSIS_PARAMETERS = {
    "search_cdf_min": 0.8, "search_cdf_max": 0.999, "marginal_distbn_kde_bandwidth": 10.0,
    "joint_distbn_kde_bandwidth": 5.0, "n_hist_bins": 2048, "n_pdf_points": 256,
    "pdf_sla_min": 1, "pdf_slc_min": 1, "pdf_slt_min": 1,
    "marginal_distbn_kde_method": "opencl", "marginal_distbn_kde_kernel": "epanechnikov",
    "joint_distbn_kde_method": "opencl", "joint_distbn_kde_kernel": "gaussian",
    "do_marginal_distbn_dsla": True, "do_marginal_distbn_usla": False, "do_marginal_distbn_dslt": True,
    "do_marginal_distbn_uslt": False, "do_marginal_distbn_dslc": True, "do_marginal_distbn_uslc": False,
    "do_joint_distribn_dsla_dslt": True, "do_joint_distribn_usla_uslt": False,
    "do_joint_distribn_uslt_dslt": False, "do_joint_distribn_dsla_usla": False,
    "do_joint_distribn_dsla_dslc": True, "do_joint_distribn_dslt_dslc": True,
    "do_joint_distribn_usla_uslc": False, "do_joint_distribn_uslc_dslc": False,
}

# name: (x field, y field, x direction, y direction, log-limit parameters), as
# the reference's compute_marginal_distribn_* / compute_joint_distribn_*
# methods choose them (analysis.py:191-573), in the order do() runs them
_SLA_SLC = ("pdf_sla_min", "pdf_sla_max", "pdf_slc_min", "pdf_slc_max")
_SLT_SLA = ("pdf_slt_min", "pdf_slt_max", "pdf_sla_min", "pdf_sla_max")
_SLC_SLA = ("pdf_slc_min", "pdf_slc_max", "pdf_sla_min", "pdf_sla_max")
MARGINALS = [("dsla", "sla", "slc", 0, 0, _SLA_SLC), ("usla", "sla", "slc", 1, 1, _SLA_SLC),
             ("dslt", "slt", "sla", 0, 0, _SLT_SLA), ("uslt", "slt", "sla", 1, 1, _SLT_SLA),
             ("dslc", "slc", "sla", 0, 0, _SLC_SLA), ("uslc", "slc", "sla", 1, 1, _SLC_SLA)]
JOINTS = [("dsla_usla", "sla", "sla", 0, 1, ("pdf_sla_min", "pdf_sla_max", "pdf_sla_min", "pdf_sla_max")),
          ("usla_uslt", "sla", "slt", 1, 1, ("pdf_sla_min", "pdf_sla_max", "pdf_slt_min", "pdf_slt_max")),
          # the reference pairs slt (x) with sla (y) here, under sla-then-slt limits
          ("dsla_dslt", "slt", "sla", 0, 0, ("pdf_sla_min", "pdf_sla_max", "pdf_slt_min", "pdf_slt_max")),
          ("dslt_dslc", "slt", "slc", 0, 0, ("pdf_slt_min", "pdf_slt_max", "pdf_slc_min", "pdf_slc_max")),
          ("uslt_dslt", "slt", "slt", 1, 0, ("pdf_slt_min", "pdf_slt_max", "pdf_slt_min", "pdf_slt_max")),
          ("usla_uslc", "sla", "slc", 1, 1, _SLA_SLC),
          ("dsla_dslc", "sla", "slc", 0, 0, _SLA_SLC),
          ("uslc_dslc", "slc", "slc", 1, 0, ("pdf_slc_min", "pdf_slc_max", "pdf_slc_min", "pdf_slc_max"))]


class Analysis:
    """``streamlines.analysis.Analysis`` (analysis.py:40-577) over the device
    KDE: ``do()`` computes the marginal pdfs (``mpdf_<name>``: modes,
    statistics, channel threshold) and the joint pdfs (``jpdf_<name>``: mode)
    that the job's ``do_*`` flags select, from ``trace``'s slc/slt/sla, or
    from ``data`` when a method is given one.  Only the 'opencl' KDE method
    exists here (on the GPU); the reference's scipy/sklearn alternatives and
    its elevation / slope pdfs (SciPy's gaussian_kde on the host, outside the
    KDE path) are not restated."""

    def __init__(self, state, imported_parameters, geodata, preprocess, trace):
        params = dict(ANALYSIS_PARAMETERS)
        if imported_parameters:
            params.update(imported_parameters.get("analysis", imported_parameters))
        for k, v in params.items():
            setattr(self, k, v)
        self.state, self.geodata, self.preprocess, self.trace = state, geodata, preprocess, trace
        self.mapping = None
        self.area_correction_factor = 1.0
        self.length_correction_factor = 1.0

    def _augment(self, mapping):
        self.mapping = mapping

    def print(self, *args, **kwargs):
        vprint(getattr(self.state, "verbose", False), *args, **kwargs)

    def do(self):
        self.print("\n**Analysis begin**")
        for name, *_ in MARGINALS:
            if getattr(self, "do_marginal_distbn_" + name, False):
                getattr(self, "compute_marginal_distribn_" + name)()
        for name, *_ in JOINTS:
            if getattr(self, "do_joint_distribn_" + name, False):
                getattr(self, "compute_joint_distribn_" + name)()
        self.print("**Analysis end**\n")

    def estimate_channel_threshold(self, data, verbose=None):
        """analysis.py:120-134: the dslt threshold, None when none qualifies."""
        try:
            self.compute_marginal_distribn_dslt(data)
            return self.mpdf_dslt.channel_threshold_x
        except AttributeError as error:
            self.print("Failed to estimate channel threshold:", error)
            return None

    def _get_limits(self, attr_list):
        return [np.log(getattr(self, a)) if hasattr(self, a) and getattr(self, a) is not None else None
                for a in attr_list]

    def _method(self, key):
        method = getattr(self, key)
        if method != "opencl":
            raise NotImplementedError('KDE method "{}": only "opencl" (the device KDE) is built'.format(method))

    def _arrays(self, data, fx, fy):
        src = data if data is not None else self.trace
        return getattr(src, fx + "_array"), getattr(src, fy + "_array"), (data.mask_array if data is not None
                                                                           else None)

    def compute_marginal_distribn(self, x_array, y_array, mask_array=None, up_down_idx_x=0, up_down_idx_y=0,
                                  n_hist_bins=None, n_pdf_points=None, kernel=None, bandwidth=None, method=None,
                                  logx_min=None, logy_min=None, logx_max=None, logy_max=None):
        if method is None:
            self._method("marginal_distbn_kde_method")
        elif method != "opencl":
            raise NotImplementedError('KDE method "{}": only "opencl" (the device KDE) is built'.format(method))
        return compute_marginal_distribn(
            x_array, y_array, mask_array, up_down_idx_x, up_down_idx_y,
            n_hist_bins=n_hist_bins or self.n_hist_bins, n_pdf_points=n_pdf_points or self.n_pdf_points,
            kernel=kernel or self.marginal_distbn_kde_kernel,
            bandwidth=bandwidth if bandwidth is not None else self.marginal_distbn_kde_bandwidth,
            logx_min=logx_min, logy_min=logy_min, logx_max=logx_max, logy_max=logy_max,
            search_cdf_min=self.search_cdf_min, search_cdf_max=self.search_cdf_max,
            pixel_size=getattr(self.geodata, "roi_pixel_size", None),
            cl_platform=getattr(self.state, "cl_platform", 0), cl_device=getattr(self.state, "cl_device", 0),
            verbose=getattr(self.state, "verbose", False))

    def compute_joint_distribn(self, x_array, y_array, mask_array=None, up_down_idx_x=0, up_down_idx_y=0,
                               n_hist_bins=None, n_pdf_points=None, thresholding_marginal_distbn=None,
                               kernel=None, bandwidth=None, method=None, logx_min=None, logy_min=None,
                               logx_max=None, logy_max=None, upstream_modal_length=None):
        if method is None:
            self._method("joint_distbn_kde_method")
        elif method != "opencl":
            raise NotImplementedError('KDE method "{}": only "opencl" (the device KDE) is built'.format(method))
        return compute_joint_distribn(
            x_array, y_array, mask_array, up_down_idx_x, up_down_idx_y,
            n_hist_bins=n_hist_bins or self.n_hist_bins, n_pdf_points=n_pdf_points or self.n_pdf_points,
            kernel=kernel or self.joint_distbn_kde_kernel,
            bandwidth=bandwidth if bandwidth is not None else self.joint_distbn_kde_bandwidth,
            logx_min=logx_min, logy_min=logy_min, logx_max=logx_max, logy_max=logy_max,
            pixel_size=getattr(self.geodata, "roi_pixel_size", None),
            cl_platform=getattr(self.state, "cl_platform", 0), cl_device=getattr(self.state, "cl_device", 0),
            verbose=getattr(self.state, "verbose", False))


def _marginal_method(name, fx, fy, ix, iy, limits):
    def method(self, data=None):
        x_array, y_array, mask_array = self._arrays(data, fx, fy)
        if name == "usla":
            mask_array = data.mask_array  # the reference reads it whether or not data is given
        lx0, lx1, ly0, ly1 = self._get_limits(limits)
        setattr(self, "mpdf_" + name, self.compute_marginal_distribn(
            x_array, y_array, mask_array, up_down_idx_x=ix, up_down_idx_y=iy,
            logx_min=lx0, logy_min=ly0, logx_max=lx1, logy_max=ly1))
    method.__name__ = "compute_marginal_distribn_" + name
    method.__doc__ = "The marginal pdf '{}' (analysis.py:191-323).".format(name)
    return method


def _joint_method(name, fx, fy, ix, iy, limits):
    def method(self, data=None):
        x_array, y_array, mask_array = self._arrays(data, fx, fy)
        lx0, lx1, ly0, ly1 = self._get_limits(limits)
        setattr(self, "jpdf_" + name, self.compute_joint_distribn(
            x_array, y_array, mask_array, up_down_idx_x=ix, up_down_idx_y=iy,
            thresholding_marginal_distbn=getattr(self, "mpdf_dsla", None),
            logx_min=lx0, logy_min=ly0, logx_max=lx1, logy_max=ly1))
    method.__name__ = "compute_joint_distribn_" + name
    method.__doc__ = "The joint pdf '{}' (analysis.py:383-573).".format(name)
    return method


for _row in MARGINALS:
    setattr(Analysis, "compute_marginal_distribn_" + _row[0], _marginal_method(*_row))
for _row in JOINTS:
    setattr(Analysis, "compute_joint_distribn_" + _row[0], _joint_method(*_row))
del _row
