"""Fast-marching hillslope lengths of pass 2 (the reference's
``Mapping.fmm_lengths``, python/streamlines/mapping.py:841-900).

For every selected fine subsegment s the reference builds phi on the
window -- +1 on the pixels with |label| == |s| grown by one pixel
(4-neighbour dilation), -1 on its own thin-channel pixels, masked elsewhere
-- asks scikit-fmm for the signed distance from phi's zero contour (``dx`` =
the pixel size) and keeps twice the mean distance, truncated into its int32
result array, when the subsegment has more than 4 pixels per channel pixel.

Here the distances come from a solver that takes every distinct |s| of a
window at once and returns per problem the sum and count of the reached
distances and the two pixel counts; the default one is the CUDA kernel
``slm_fmm_lengths`` (one thread per subsegment, each over the box of its
grown region).  This module keeps the reference's call-site rules on top:
the selection, the ratio test, the mean as sum / count times 2, the int32
truncation, and "no zero contour" leaving a 0 (the reference catches
skfmm's exception).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib

STATUS_OK, STATUS_NO_CHANNEL, STATUS_NO_CONTOUR = 0, 1, 2


def _boxes(label_abs, keys):
    """Per key (sorted 1-D int64 tensor): x0, x1, y0, y1 of the pixels with
    that |label|, grown by one and clipped to the grid; rows with no pixel
    have x0 > x1."""
    nx, ny = label_abs.shape
    n = keys.numel()
    dev = label_abs.device
    flat = label_abs.reshape(-1).to(torch.int64)
    k = torch.searchsorted(keys, flat).clamp_(max=n - 1)
    hit = keys[k] == flat
    idx = k[hit]
    pos = torch.nonzero(hit).squeeze(1)
    xs, ys = pos // ny, pos % ny
    big = torch.iinfo(torch.int64).max
    lo_x = torch.full((n,), big, dtype=torch.int64, device=dev).scatter_reduce_(0, idx, xs, "amin")
    hi_x = torch.full((n,), -1, dtype=torch.int64, device=dev).scatter_reduce_(0, idx, xs, "amax")
    lo_y = torch.full((n,), big, dtype=torch.int64, device=dev).scatter_reduce_(0, idx, ys, "amin")
    hi_y = torch.full((n,), -1, dtype=torch.int64, device=dev).scatter_reduce_(0, idx, ys, "amax")
    b = torch.stack([lo_x, hi_x, lo_y, hi_y], 1).cpu().numpy()
    empty = b[:, 1] < 0
    b[:, 0] = np.maximum(b[:, 0] - 1, 0)
    b[:, 1] = np.minimum(b[:, 1] + 1, nx - 1)
    b[:, 2] = np.maximum(b[:, 2] - 1, 0)
    b[:, 3] = np.minimum(b[:, 3] + 1, ny - 1)
    b[empty] = (1, 0, 1, 0)
    return b


def device_solver(label, flags, thin_bit, subsegments, dx, order, fields=False):
    """Per |label| value in ``subsegments`` (int array): (sum, count, n_phi,
    n_channel, status) NumPy arrays from ``slm_fmm_lengths``.  ``label``
    (int32) and ``flags`` (uint32 values) are [nx, ny] tensors on the GPU.
    With ``fields`` a sixth item lists per problem (box, signed distance
    times dx on the box, reached mask)."""
    dev = label.device
    nx, ny = label.shape
    keys = np.asarray(subsegments, dtype=np.int64)
    n = keys.shape[0]
    out = [np.zeros(n, np.float64), np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int64),
           np.full(n, STATUS_NO_CHANNEL, np.int32)]
    if n == 0:
        return tuple(out) + (([],) if fields else ())
    label = label.to(torch.int32).contiguous()
    flags32 = flags.to(torch.int64).bitwise_and(0xFFFFFFFF).to(torch.int32).contiguous()
    boxes = _boxes(label.abs(), torch.from_numpy(keys).to(dev))
    live = boxes[:, 1] >= boxes[:, 0]
    li = np.nonzero(live)[0]
    if li.size:
        b = boxes[li]
        areas = (b[:, 1] - b[:, 0] + 1) * (b[:, 3] - b[:, 2] + 1)
        offs = np.concatenate([[0], np.cumsum(areas)[:-1]]).astype(np.int64)
        total = int(areas.sum())
        m = li.size
        val = torch.empty(total, dtype=torch.float64, device=dev)
        st = torch.empty(total, dtype=torch.uint8, device=dev)
        hkey = torch.empty(4 * total, dtype=torch.float64, device=dev)
        hidx = torch.empty(4 * total, dtype=torch.int32, device=dev)
        # inputs up in one buffer (offsets int64, boxes and labels int32),
        # outputs back in one (sum f64, count / n_phi / n_channel i64, status i32)
        up = np.empty(8 * m + 16 * m + 4 * m, dtype=np.uint8)
        up[:8 * m].view(np.int64)[:] = offs
        up[8 * m:24 * m].view(np.int32)[:] = b.astype(np.int32).reshape(-1)
        up[24 * m:].view(np.int32)[:] = keys[li].astype(np.int32)
        up_d = torch.from_numpy(up).to(dev)
        down_d = torch.empty(36 * m, dtype=torch.uint8, device=dev)
        P = _lib.ptr
        u0, d0 = up_d.data_ptr(), down_d.data_ptr()

        def at(base, byte):
            return ctypes.c_void_p(base + byte)
        _lib.check(_lib.load().slm_fmm_lengths(
            P(label), P(flags32), int(nx), int(ny), int(thin_bit) & 0xFFFFFFFF, at(u0, 24 * m), at(u0, 8 * m),
            at(u0, 0), int(m), total, int(order), float(dx), P(val), P(st), P(hkey), P(hidx), at(d0, 0),
            at(d0, 8 * m), at(d0, 16 * m), at(d0, 24 * m), at(d0, 32 * m),
            torch.cuda.current_stream(dev).cuda_stream))
        down = down_d.cpu().numpy()
        out[0][li] = down[:8 * m].view(np.float64)
        for k in range(3):
            out[1 + k][li] = down[8 * m * (k + 1):8 * m * (k + 2)].view(np.int64)
        out[4][li] = down[32 * m:].view(np.int32)
        if fields:
            vh, sh = val.cpu().numpy(), st.cpu().numpy()
            per = [None] * n
            for j, i in enumerate(li):
                x0, x1, y0, y1 = (int(v) for v in b[j])
                a = slice(int(offs[j]), int(offs[j] + areas[j]))
                shape = (x1 - x0 + 1, y1 - y0 + 1)
                per[i] = ((x0, x1, y0, y1), vh[a].reshape(shape), (sh[a] & 3).reshape(shape) == 2)
            out.append(per)
    elif fields:
        out.append([None] * n)
    bad = (out[4] > STATUS_NO_CONTOUR)
    if bad.any():
        raise RuntimeError("slm_fmm_lengths: problem status {} (subsegment {})".format(
            int(out[4][bad][0]), int(keys[bad][0])))
    return tuple(out)


def fmm_lengths(label, flags, thin_bit, selected, dx, order=2, solver=None):
    """The reference's ``fmm_lengths`` result for the ``selected`` fine
    labels (signed, nonzero, in the reference's order): an int32 array, 0
    where the subsegment was skipped.  ``label`` / ``flags`` are the
    window's [nx, ny] grids (tensors on the GPU for the default solver)."""
    selected = np.asarray(selected, dtype=np.int32)
    hsl = np.zeros(selected.shape[0], dtype=np.int32)
    if selected.size == 0:
        return hsl
    keys = np.unique(np.abs(selected.astype(np.int64)))
    sums, counts, n_phi, n_chan, status = (solver or device_solver)(label, flags, thin_bit, keys, dx, order)[:5]
    at = np.searchsorted(keys, np.abs(selected.astype(np.int64)))
    for i, k in enumerate(at):
        if status[k] != STATUS_OK or n_chan[k] == 0:
            continue  # no channel pixel, or no zero contour (skfmm raises; the reference passes)
        ratio = int(n_phi[k]) / int(n_chan[k])
        mean = np.float64(sums[k]) * 1.0 / np.int64(counts[k])
        value = mean * 2.0
        if ratio > 4.0:
            hsl[i] = np.array([value], dtype=np.float64).astype(np.int32)[0]
    return hsl
