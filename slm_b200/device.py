"""Device selection and host<->device staging for the stage wrappers."""
from __future__ import annotations

import os

import numpy as np
import torch

from . import _lib


def cuda_device(cl_platform=0, cl_device=0):
    """CUDA device standing in for the reference's (cl_platform, cl_device) pair.

    The reference picks an OpenCL device by index (pocl.py:76-93); here the
    index selects a CUDA device modulo the number present.  Raises if none is.
    """
    _lib.load()
    n = torch.cuda.device_count()
    if n == 0 or not torch.cuda.is_available():
        raise RuntimeError("slm_b200 needs a CUDA device (B200, sm_100a); none is visible")
    idx = int(cl_device or 0) % n
    return torch.device("cuda", idx)


def to_device(array, device, dtype=None):
    """Copy a NumPy array to the device; pinned-memory arrays go by async DMA."""
    a = np.ascontiguousarray(array)
    if a.dtype == np.bool_:
        a = a.view(np.uint8)
    t = torch.from_numpy(a)
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.to(device, non_blocking=t.is_pinned())


_COPY_POOL = None


def host_copy(src, min_bytes=8 << 20, pinned=False):
    """A fresh C-ordered NumPy copy of a host array (any strides, as
    ``src.copy()`` gives), split over up to 8 threads when large (np.copyto
    releases the GIL; the page faults of the new array are taken in parallel
    too).  ``pinned``: a large copy goes to page-locked memory when a GPU is
    present (torch's caching host allocator reuses it once the array is
    freed), so a later upload of it runs at DMA speed."""
    global _COPY_POOL
    src = np.asarray(src)
    if src.nbytes < min_bytes or src.ndim == 0:
        return src.copy()
    if _COPY_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _COPY_POOL = ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1)))
    dst = None
    if pinned and torch.cuda.is_available() and src.dtype in _PINNED_DTYPES:
        dst = pinned_empty(src.shape, src.dtype)
    if dst is None:
        dst = np.empty(src.shape, dtype=src.dtype)
    k = _COPY_POOL._max_workers
    if src.flags.c_contiguous:
        f, g = src.reshape(-1), dst.reshape(-1)
        n = f.size
    else:  # rows of a strided view
        f, g = src, dst
        n = src.shape[0]
    list(_COPY_POOL.map(lambda i: np.copyto(g[i * n // k:(i + 1) * n // k], f[i * n // k:(i + 1) * n // k]),
                        range(k)))
    return dst


def _parallel_copy(dst, src):
    """np.copyto of two same-size contiguous arrays, split over up to 8 threads."""
    global _COPY_POOL
    if _COPY_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _COPY_POOL = ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1)))
    f, g = src.reshape(-1), dst.reshape(-1)
    n, k = f.size, _COPY_POOL._max_workers
    list(_COPY_POOL.map(lambda i: np.copyto(g[i * n // k:(i + 1) * n // k], f[i * n // k:(i + 1) * n // k]),
                        range(k)))


_STAGING = {}


def pinned_staging(slot, shape, dtype):
    """A pinned host tensor of this shape and torch dtype, kept for reuse (one per slot)."""
    key = (slot, tuple(shape), dtype)
    st = _STAGING.get(key)
    if st is None:
        st = torch.empty(tuple(shape), dtype=dtype, pin_memory=True)
        _STAGING[key] = st
    return st


def upload(array, device, slot, dtype=None):
    """``to_device`` for large pageable arrays (any strides): gathered into a
    pinned staging buffer by several threads, cast to ``dtype`` on the way,
    then copied by DMA.  The caller synchronises the current stream before
    reusing ``slot``."""
    a = array.view(np.uint8) if array.dtype == np.bool_ else array
    dt = np.dtype(dtype) if dtype is not None else a.dtype
    if a.nbytes < (32 << 20) or a.ndim == 0:
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(device)
    st = pinned_staging(slot, a.shape, torch.from_numpy(np.empty(0, dt)).dtype)
    dst = st.numpy()
    global _COPY_POOL
    if _COPY_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _COPY_POOL = ThreadPoolExecutor(max(1, min(8, os.cpu_count() or 1)))
    n, k = a.shape[0], _COPY_POOL._max_workers
    list(_COPY_POOL.map(lambda i: np.copyto(dst[i * n // k:(i + 1) * n // k], a[i * n // k:(i + 1) * n // k],
                                            casting="unsafe"), range(k)))
    return st.to(device, non_blocking=True)


def download(tensors, slot, pinned=False):
    """Fresh NumPy copies of device tensors: all go to pinned staging buffers
    by DMA, one synchronisation, then out of them on several threads.  With
    ``pinned`` the DMA writes straight into fresh page-locked arrays that the
    caller keeps (torch's caching host allocator reuses their memory once
    they are freed), and no host copy follows."""
    if pinned and all(t.dtype in _PINNED_DTYPES.values() for t in tensors):
        outs = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in tensors]
        for o, t in zip(outs, tensors):
            o.copy_(t, non_blocking=True)
        if outs:
            torch.cuda.current_stream(tensors[0].device).synchronize()
        return [o.numpy() for o in outs]
    stages = []
    for i, t in enumerate(tensors):
        st = pinned_staging((slot, i), t.shape, t.dtype)
        st.copy_(t, non_blocking=True)
        stages.append(st)
    if stages:
        torch.cuda.current_stream(tensors[0].device).synchronize()
    return [host_copy(st.numpy()) for st in stages]


_PINNED_DTYPES = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                  np.dtype(np.uint8): torch.uint8, np.dtype(np.uint32): torch.uint32, np.dtype(np.uint16): torch.uint16,
                  np.dtype(np.int8): torch.int8, np.dtype(np.uint64): torch.uint64,
                  np.dtype(np.bool_): torch.bool}


def pinned_empty(shape, dtype):
    """A NumPy array backed by page-locked host memory (fast DMA both ways)."""
    return torch.empty(shape, dtype=_PINNED_DTYPES[np.dtype(dtype)], pin_memory=True).numpy()


def low32(t_u64):
    """Low 32 bits of a uint64 device tensor, as uint32 (the reference's wrap-around)."""
    return t_u64.view(torch.int32).view(-1, 2)[:, 0].contiguous().view(torch.uint32)


def traced(name):
    """Decorator: the call runs inside an NVTX range ``name``, so profiler
    timelines (nsys, ncu's range filters) show the stages of the path."""
    import functools

    def wrap(fn):
        @functools.wraps(fn)
        def inner(*args, **kwargs):
            with torch.cuda.nvtx.range(name):
                return fn(*args, **kwargs)
        return inner
    return wrap
