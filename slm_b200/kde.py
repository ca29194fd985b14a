"""Kernel-density estimates of log-distributions: drop-in for the reference's
``python/streamlines/kde.py``.

``estimate_univariate_pdf(distbn)`` (kde.py:116-194) and
``estimate_bivariate_pdf(distbn)`` (kde.py:35-114) keep the reference's
contract: they read the distribution object's fields (``logx_data`` or
``logxy_data``, ``n_data``, ``bandwidth``, bin and pdf spacings, ``kernel``),
set its Silverman-scaled kernel widths in log space, run histogram + smoothing
on the device (``libslm_b200.so``), and return ``(pdf, histogram)`` normalised
exactly as the reference normalises them.  The kernel parameters are the
reference's KDE macros (pocl.py:196-222).
"""
from __future__ import annotations

import numpy as np
import torch

from . import kernels
from .device import cuda_device
from .params import params_from_options, compile_options
from .useful import vprint


def kde_params(distbn, kernel_fn):
    """The KDE parameter block for one kernel, as the reference's -D macros."""
    return params_from_options(compile_options(distbn, kernel_fn, job_type="kde"))


def _device(distbn):
    return cuda_device(getattr(distbn, "cl_platform", 0) or 0, getattr(distbn, "cl_device", 0) or 0)


def prepare_univariate(distbn):
    """Silverman-scaled kernel width in log space (kde.py:151-158)."""
    stddev_x = np.std(distbn.logx_data)
    distbn.kdf_width_x = 1.06 * stddev_x * np.power(distbn.n_data, -0.2) * distbn.bandwidth
    distbn.kdf_width_y = 0.0
    distbn.n_kdf_part_points_x = np.uint32(np.floor(distbn.kdf_width_x / distbn.pdf_dx)) // 2
    distbn.n_kdf_part_points_y = 0


def prepare_bivariate(distbn):
    """Kernel widths of both axes (kde.py:71-82)."""
    sl_array = distbn.logxy_data
    stddev_x = np.std(sl_array[:, 0])
    stddev_y = np.std(sl_array[:, 1])
    distbn.kdf_width_x = 1.06 * stddev_x * np.power(distbn.n_data, -0.2) * distbn.bandwidth
    distbn.kdf_width_y = 1.06 * stddev_y * np.power(distbn.n_data, -0.2) * distbn.bandwidth
    distbn.n_kdf_part_points_x = (np.uint32(np.floor(distbn.kdf_width_x / distbn.bin_dx)) // 2)
    distbn.n_kdf_part_points_y = (np.uint32(np.floor(distbn.kdf_width_y / distbn.bin_dy)) // 2)


def estimate_univariate_pdf(distbn, do_detrend=False, logx_vec=None):
    verbose = getattr(distbn, "verbose", False)
    vprint(verbose, "Estimating univariate pdf...", end="")
    dev = _device(distbn)
    sl_array = distbn.logx_data
    bin_dx = distbn.bin_dx
    prepare_univariate(distbn)
    prm = kde_params(distbn, "histogram_univariate")
    nb, npp = int(distbn.n_hist_bins), int(distbn.n_pdf_points)
    with torch.cuda.device(dev):
        data_d = torch.from_numpy(np.ascontiguousarray(sl_array, dtype=np.float32).reshape(-1)).to(dev)
        hist_d = torch.zeros(nb, dtype=torch.uint32, device=dev)
        kernels.histogram_univariate(prm, data_d, hist_d)
        histogram_array = hist_d.cpu().numpy().reshape(nb, 1)
        if do_detrend:
            from scipy.stats import norm
            x = logx_vec
            pdf = histogram_array.copy().astype(np.float32)
            mean = (np.sum(x * pdf) / np.sum(pdf))
            stddev = np.sqrt(np.sum((x - mean) ** 2 * pdf) / np.sum(pdf))
            pdf /= norm.pdf(logx_vec, mean, stddev)
            pdf /= np.sum(pdf)
            pdf *= np.sum(histogram_array)
            histogram_array = pdf.copy().astype(np.uint32)
            hist_d = torch.from_numpy(np.ascontiguousarray(histogram_array).reshape(-1)).to(dev)
        pdf_d = torch.zeros(npp, dtype=torch.float32, device=dev)
        kernels.pdf_univariate(kde_params(distbn, "pdf_univariate"), hist_d, pdf_d)
        pdf_array = pdf_d.cpu().numpy().reshape(npp, 1)
    vprint(verbose, "done")
    # the reference normalises by Python's builtin sum over the rows: a
    # left-to-right sum in the array's own dtype, which accumulate gives
    return (pdf_array / (_row_sum(pdf_array) * bin_dx),
            histogram_array / (_row_sum(histogram_array) * bin_dx))


def _row_sum(a):
    """``sum(a)`` (builtin) of an [n, 1] array: the rows added left to right in
    a's dtype (kde.py:193-194)."""
    if a.shape[0] == 0:
        return 0
    return np.add.accumulate(a, axis=0, dtype=a.dtype)[-1]


def estimate_bivariate_pdf(distbn):
    verbose = getattr(distbn, "verbose", False)
    vprint(verbose, "Estimating bivariate pdf...", end="")
    dev = _device(distbn)
    sl_array = distbn.logxy_data
    bin_dx, bin_dy = distbn.bin_dx, distbn.bin_dy
    prepare_bivariate(distbn)
    nb, npp = int(distbn.n_hist_bins), int(distbn.n_pdf_points)
    with torch.cuda.device(dev):
        data_d = torch.from_numpy(np.ascontiguousarray(sl_array, dtype=np.float32)).to(dev)
        hist_d = torch.zeros(nb * nb, dtype=torch.uint32, device=dev)
        kernels.histogram_bivariate(kde_params(distbn, "histogram_bivariate"), data_d, hist_d)
        part_d = torch.zeros(nb * nb, dtype=torch.float32, device=dev)
        kernels.pdf_bivariate_rows(kde_params(distbn, "pdf_bivariate_rows"), hist_d, part_d)
        pdf_d = torch.zeros(npp * npp, dtype=torch.float32, device=dev)
        kernels.pdf_bivariate_cols(kde_params(distbn, "pdf_bivariate_cols"), part_d, pdf_d)
        histogram_array = hist_d.cpu().numpy().reshape(nb, nb)
        pdf_array = pdf_d.cpu().numpy().reshape(npp, npp)
    vprint(verbose, "done")
    return (pdf_array / (np.sum(pdf_array) * bin_dx * bin_dy),
            histogram_array / (np.sum(histogram_array) * bin_dx * bin_dy))
