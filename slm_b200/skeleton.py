"""Binary thinning used between the channel-mapping kernels.

The reference thins the channel mask on the host with scikit-image,
``skeletonize(medial_axis(channel_array))`` (mapping.py:707-719).  scikit-image
is not available here, so this module provides the project's own host-side
thinning: the Zhang-Suen parallel thinning algorithm (T. Y. Zhang and
C. Y. Suen, "A fast parallel algorithm for thinning digital patterns",
CACM 27(3), 1984), vectorised with NumPy.  Its output is a one-pixel-wide,
8-connected skeleton like skimage's, but not the same pixels: parity of this
host step with the reference is unpinned, so the kernels after it are
compared with the oracle on identical thinned inputs.
"""
from __future__ import annotations

import numpy as np


def _neighbours(img):
    p = np.pad(img, 1)
    # P2..P9 clockwise from north (x is the first axis, so "north" is -x)
    return [p[:-2, 1:-1], p[:-2, 2:], p[1:-1, 2:], p[2:, 2:],
            p[2:, 1:-1], p[2:, :-2], p[1:-1, :-2], p[:-2, :-2]]


def zhang_suen(mask, max_iter=10000):
    """Thin a boolean image to a one-pixel-wide skeleton."""
    img = np.ascontiguousarray(mask, dtype=np.uint8).copy()
    for _ in range(max_iter):
        changed = False
        for step in (0, 1):
            n = _neighbours(img)
            b = sum(n)
            seq = n + [n[0]]
            a = sum(((seq[k] == 0) & (seq[k + 1] == 1)).astype(np.uint8) for k in range(8))
            p2, p4, p6, p8 = n[0], n[2], n[4], n[6]
            if step == 0:
                c1 = (p2 * p4 * p6) == 0
                c2 = (p4 * p6 * p8) == 0
            else:
                c1 = (p2 * p4 * p8) == 0
                c2 = (p2 * p6 * p8) == 0
            rm = (img == 1) & (b >= 2) & (b <= 6) & (a == 1) & c1 & c2
            if rm.any():
                img[rm] = 0
                changed = True
        if not changed:
            break
    return img.astype(bool)


def zhang_suen_device(mask, max_iter=10000, device=None):
    """The same thinning on the GPU (``slm_thin``): identical output."""
    import ctypes

    import torch

    from . import _lib
    from .device import cuda_device
    dev = device if device is not None else cuda_device(0, 0)
    img = np.ascontiguousarray(mask, dtype=np.uint8)
    nx, ny = img.shape
    with torch.cuda.device(dev):
        d = torch.from_numpy(img).to(dev)
        scratch = torch.empty_like(d)
        flag = torch.zeros(1, dtype=torch.int32, device=dev)
        it = ctypes.c_uint32(0)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(_lib.load().slm_thin(_lib.ptr(d), _lib.ptr(scratch), nx, ny, int(max_iter), _lib.ptr(flag),
                                        ctypes.byref(it), stream))
        return d.cpu().numpy().astype(bool)
