"""DTM preprocessing on the GPU: the conditioned gradient vector field.

Mirrors ``streamlines.preprocess.Preprocess`` (python/streamlines/
preprocess.py:479-699).  The reference conditions the DTM on the host:

- ``find_blockages`` (:647-699): two scipy ``generic_filter`` passes with
  Python callbacks;
- ``compute_topo_gradient_field`` / ``compute_gradient_velocity_field``
  (:51-63, :176-193): NumPy;
- ``find_and_fix_loops`` (:302-349) and ``fix_blockages`` (:351-387): numba
  loops;
- the renormalisation, edge padding (:588-598) and ``mask_nan_uv``
  (:602-621).

All of it runs here as one kernel, ``slm_preprocess``, with the same results
bit for bit (the slope, an arctangent, within float32 rounding).  The
outputs can stay on the device for the tracer (``download=False``).

The reference's unconditioned path (``raw_gradient_vector_field``,
:623-645) calls a function ``derivatives`` that the package does not define,
so it cannot run; ``Preprocess.do`` raises for it in the same place.
"""
from __future__ import annotations

import ctypes
import types

import numpy as np
import torch

from . import _lib
from ._lib import SlmPreprocessParams, check, ptr
from .device import cuda_device, traced

DEFAULTS = {"do_normalize_speed": True, "vecsum_threshold": 0.95, "divergence_threshold": -0.5,
            "curl_threshold": 0.0}


def _where(a):
    """np.where of a 2-D array as an [n, 2] (x, y) array (preprocess.py:676-683)."""
    w = np.where(a)
    return np.stack((w[0], w[1])).T


def conditioned_gradient_vector_field(roi, pixel_size, pad_width, vecsum_threshold=0.95,
                                      divergence_threshold=-0.5, curl_threshold=0.0,
                                      do_normalize_speed=True, device=None, download=True, stream=None):
    """Condition one ROI ([nx, ny] float32 or float64, x-major, NaN = no data).

    Returns a namespace with the reference's arrays: ``uv_array`` [nxp, nyp, 2]
    float32 (NaN vectors zeroed), ``slope_array``, ``uv_mask_array`` (the 'uv'
    active mask), ``mask_array`` (pad frame | NaN ROI | uv_mask),
    ``blockages_array``, ``blocked_neighbors_array``, ``where_blockages_array``,
    ``where_blocked_neighbors_array``, ``where_looped_array``, ``n_loops``,
    ``roi_gradx_array``, ``roi_grady_array``.  With ``download=False`` the
    grids are CUDA tensors (masks uint8), the looped-cell count stays on the
    device (``n_loop_cells``, int32; n_loops is 4x) and nothing synchronises."""
    L = _lib.load()
    dev = device if device is not None else cuda_device(0, 0)
    if isinstance(roi, torch.Tensor):
        if roi.dim() != 2 or roi.dtype not in (torch.float32, torch.float64):
            raise ValueError("roi must be a 2-D float32 or float64 tensor")
        roi_d = roi.to(dev).contiguous()
    else:
        a = np.asarray(roi)
        if a.ndim != 2:
            raise ValueError("roi must be 2-D")
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        roi_d = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    nx, ny = roi_d.shape
    if nx < 2 or ny < 2:
        raise ValueError("Shape of array too small to calculate a numerical gradient, "
                         "at least 2 elements are required along each axis")
    pw = int(pad_width)
    nxp, nyp = nx + 2 * pw, ny + 2 * pw
    prm = SlmPreprocessParams(float(pixel_size), float(vecsum_threshold), float(divergence_threshold),
                              float(curl_threshold), pw, 1 if do_normalize_speed else 0)
    with torch.cuda.device(dev):
        f32, u8 = torch.float32, torch.uint8
        uv = torch.empty((nxp, nyp, 2), dtype=f32, device=dev)
        slope = torch.empty((nxp, nyp), dtype=f32, device=dev)
        uv_mask = torch.empty((nxp, nyp), dtype=u8, device=dev)
        mask = torch.empty((nxp, nyp), dtype=u8, device=dev)
        blk = torch.empty((nx, ny), dtype=u8, device=dev)
        nbr = torch.empty((nx, ny), dtype=u8, device=dev)
        cells = torch.empty((nx, ny), dtype=u8, device=dev)
        gx = torch.empty((nx, ny), dtype=f32, device=dev)
        gy = torch.empty((nx, ny), dtype=f32, device=dev)
        n_cells = torch.zeros(1, dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(L.slm_preprocess(ptr(roi_d), 1 if roi_d.dtype == torch.float64 else 0, nx, ny, ctypes.byref(prm),
                               ptr(uv), ptr(slope), ptr(uv_mask), ptr(mask), ptr(blk), ptr(nbr), ptr(cells),
                               ptr(gx), ptr(gy), ptr(n_cells), ctypes.c_void_p(s.cuda_stream)))
        if not download:
            return types.SimpleNamespace(uv_array=uv, slope_array=slope, uv_mask_array=uv_mask, mask_array=mask,
                                         blockages_array=blk, blocked_neighbors_array=nbr, loop_cells=cells,
                                         n_loop_cells=n_cells, roi_gradx_array=gx, roi_grady_array=gy)
        cells_h = cells.cpu().numpy()
        cx, cy = np.nonzero(cells_h)
        where_looped = np.zeros((4 * cx.size, 2), np.uint32)
        for k, (ox, oy) in enumerate(((0, 0), (1, 0), (0, 1), (1, 1))):
            where_looped[k::4, 0] = cx + ox
            where_looped[k::4, 1] = cy + oy
        blk_h, nbr_h = blk.cpu().numpy(), nbr.cpu().numpy()
        return types.SimpleNamespace(
            uv_array=uv.cpu().numpy(), slope_array=slope.cpu().numpy(),
            uv_mask_array=uv_mask.cpu().numpy().astype(bool), mask_array=mask.cpu().numpy().astype(bool),
            blockages_array=blk_h, blocked_neighbors_array=nbr_h,
            where_blockages_array=_where(blk_h), where_blocked_neighbors_array=_where(nbr_h),
            loop_cells=cells_h, where_looped_array=where_looped, n_loops=int(4 * cx.size),
            roi_gradx_array=gx.cpu().numpy(), roi_grady_array=gy.cpu().numpy())


class Preprocess:
    """``streamlines.preprocess.Preprocess`` with the conditioning on the GPU.

    ``imported_parameters``: the job's parameter dictionary (its
    'preprocess' section, or that section itself); ``geodata``: an object
    with ``roi_array``, ``pixel_size`` and ``pad_width`` (as the reference's
    Geodata); ``state``: an object with ``do_condition`` and, optionally,
    ``add_active_mask`` (called with {'uv': mask} as mask_nan_uv does)."""

    def __init__(self, state, imported_parameters, geodata, device=None):
        params = dict(DEFAULTS)
        sec = imported_parameters.get("preprocess", imported_parameters) if imported_parameters else {}
        params.update({k: v for k, v in sec.items() if k in DEFAULTS or k == "do_simple_gradient_vector_field"})
        for k, v in params.items():
            setattr(self, k, v)
        self.state, self.geodata, self.device = state, geodata, device

    @traced("slm.Preprocess.do")
    def do(self):
        if getattr(self.state, "do_condition", True):
            self.conditioned_gradient_vector_field()
        else:
            self.raw_gradient_vector_field()
        self.mask_nan_uv()

    def conditioned_gradient_vector_field(self):
        g = self.geodata
        r = conditioned_gradient_vector_field(g.roi_array, g.pixel_size, g.pad_width, self.vecsum_threshold,
                                              self.divergence_threshold, self.curl_threshold,
                                              self.do_normalize_speed, device=self.device)
        for k in ("uv_array", "slope_array", "blockages_array", "blocked_neighbors_array", "where_blockages_array",
                  "where_blocked_neighbors_array", "where_looped_array", "n_loops", "roi_gradx_array",
                  "roi_grady_array", "mask_array"):
            setattr(self, k, getattr(r, k))
        self._uv_mask = r.uv_mask_array

    def mask_nan_uv(self):
        """The NaN vectors are zeroed on the device; this registers the mask."""
        add = getattr(self.state, "add_active_mask", None)
        if add is not None:
            add({"uv": self._uv_mask})
        self.uv_mask_array = self._uv_mask

    def raw_gradient_vector_field(self):
        raise NameError("name 'derivatives' is not defined (the reference's unconditioned path, "
                        "preprocess.py:623-645, calls a function its package does not define)")
