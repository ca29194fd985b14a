"""Device execution of one mapping kernel on NumPy buffers (the reference's
per-call contract, pocl.gpu_compute, pocl.py:503-560: copy the buffers to the
device, run, copy the written ones back)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, ptr, sref
from .device import cuda_device

# kernel -> (entry point, indices of the buffers it writes, extra arguments)
SPECS = {
    "connect_channels": ("slm_connect_channels", (2,), "status"),
    "map_channel_heads": ("slm_map_channel_heads", (2,), None),
    "prune_channel_heads": ("slm_prune_channel_heads", (2,), None),
    "count_downchannels": ("slm_count_downchannels", (2, 3, 4), "workspace"),
    "flag_downchannels": ("slm_flag_downchannels", (2, 3), "workspace"),
    "label_confluences": ("slm_label_confluences", (3,), None),
    "segment_downchannels": ("slm_segment_downchannels", (2, 5), "status"),
    "segment_hillslopes": ("slm_segment_hillslopes", (5,), None),
    "subsegment_channel_edges": ("slm_subsegment_channel_edges", (2, 5), "status"),
    "subsegment_flanks": ("slm_subsegment_flanks", (5,), None),
    "fix_right_flanks": ("slm_fix_right_flanks", (5,), "workspace"),
    "fix_left_flanks": ("slm_fix_left_flanks", (5,), "workspace"),
    "hillslopes": ("slm_hillslopes", (4,), None),
    "hillslope_lengths": ("slm_hillslope_lengths", (4,), None),
}
# bytes of the flank path store.  None: 2 KiB per item (at least 1 GiB), at
# most half the device's free memory and FLANK_PATH_MAX.  The walks are
# traced once into it when they fit (~45 GB at 8192^2); otherwise they are
# traced again into index-ordered chunks of it.  The free memory is asked
# for (cudaMemGetInfo, milliseconds a call) only above the 1 GiB floor, or
# when the floor itself cannot be allocated: not per call of a small window.
FLANK_PATH_BUDGET = None
FLANK_PATH_MAX = 96 << 30
_MIN_WS = {
    "count_downchannels": lambda L, p, n: L.slm_count_downchannels_workspace(n, 0),
    "flag_downchannels": lambda L, p, n: L.slm_flag_downchannels_workspace(n, p.nxy_padded),
    "fix_right_flanks": lambda L, p, n: L.slm_fix_flanks_workspace(n, p.nxy_padded, 0),
    "fix_left_flanks": lambda L, p, n: L.slm_fix_flanks_workspace(n, p.nxy_padded, 0),
}


def _to_dev(a, dev):
    a = np.ascontiguousarray(a)
    if a.dtype == np.bool_:
        a = a.view(np.uint8)
    return torch.from_numpy(a).to(dev)


def run_device(name, params, seeds_d, n, bufs, device=None, stream=None, status=None):
    """Run kernel ``name`` on device tensors (the kernel's buffers after
    ``seed_point``, in its order); returns the status word.  ``status``: a
    device uint32 word the kernel ORs its status bits into, left on the
    device (the call then returns 0 without waiting for the kernel)."""
    L = _lib.load()
    fn_name, written, extra = SPECS[name]
    fn = getattr(L, fn_name)
    dev = device if device is not None else cuda_device(0, 0)
    st = stream if stream is not None else ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    args = [sref(params), int(n), ptr(seeds_d)] + [ptr(b) for b in bufs]
    keep = status is not None
    if not keep:
        status = torch.zeros(1, dtype=torch.uint32, device=dev)
    if extra == "status":
        check(fn(*(args + [ptr(status), st])))
    elif extra == "workspace":
        need = ctypes.c_uint64(0)
        size = int(_MIN_WS[name](L, params, n))
        if name.startswith("fix_"):
            # the flank fix stores paths chunk by chunk within this budget
            budget = FLANK_PATH_BUDGET
            if budget is None:
                budget = max(1 << 30, int(n) << 11)
                if budget > 1 << 30:
                    budget = min(budget, FLANK_PATH_MAX, torch.cuda.mem_get_info(dev)[0] // 2)
            try:
                ws = torch.empty(size + int(budget), dtype=torch.uint8, device=dev)
            except torch.cuda.OutOfMemoryError:
                budget = min(int(budget), torch.cuda.mem_get_info(dev)[0] // 2)
                ws = torch.empty(size + int(budget), dtype=torch.uint8, device=dev)
            size += int(budget)
        else:
            ws = torch.empty(size, dtype=torch.uint8, device=dev)
        rc = fn(*(args + [ptr(ws), size, ctypes.byref(need), st]))
        if rc == _lib.SLM_ERR_CAPACITY:
            size = int(need.value)
            ws = torch.empty(size, dtype=torch.uint8, device=dev)
            rc = fn(*(args + [ptr(ws), size, ctypes.byref(need), st]))
        check(rc)
    else:
        check(fn(*(args + [st])))
    return 0 if keep else int(status.cpu().numpy()[0])


def run(name, params, seeds, arrays, device=None):
    """Run kernel ``name`` on the device, updating the written NumPy buffers in place.
    Returns the status word (0 unless a loop cap or out-of-grid access occurred)."""
    written = SPECS[name][1]
    dev = device if device is not None else cuda_device(0, 0)
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    n = int(seeds.shape[0])
    with torch.cuda.device(dev):
        seeds_d = torch.from_numpy(seeds).to(dev) if n else torch.zeros(2, dtype=torch.float32, device=dev)
        bufs = [_to_dev(a, dev) for a in arrays]
        st = run_device(name, params, seeds_d, n, bufs, dev)
        for i in written:
            out = bufs[i].cpu().numpy()
            dst = arrays[i]
            dst[...] = out.view(dst.dtype).reshape(dst.shape) if dst.dtype != np.bool_ else out.astype(bool)
        return st
