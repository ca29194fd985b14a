"""Tensor-level calls into the C ABI (device tensors in, device tensors out).

Each function checks dtypes, devices, contiguity and sizes on the host, then
calls the ``extern "C"`` entry point on the current CUDA stream (or the one
given).  Nothing here falls back to the CPU.
"""
from __future__ import annotations

import torch

from . import _lib
from ._lib import SlmLaunch, check, ptr, sref

SCHEDULES = {"plain": _lib.SLM_SCHED_PLAIN, "persistent": _lib.SLM_SCHED_PERSISTENT}


def _need(t, dtype, numel, name):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise ValueError("{} must be a CUDA tensor".format(name))
    if t.dtype != dtype:
        raise ValueError("{} must be {}, got {}".format(name, dtype, t.dtype))
    if not t.is_contiguous():
        raise ValueError("{} must be contiguous".format(name))
    if numel is not None and t.numel() < numel:
        raise ValueError("{} has {} elements, needs {}".format(name, t.numel(), numel))


def _stream(stream):
    s = stream if stream is not None else torch.cuda.current_stream()
    return __import__("ctypes").c_void_p(s.cuda_stream)


def workspace(device=None):
    """Scratch words the field tracer needs (queue head, step/trajectory counters)."""
    n = _lib.load().slm_fields_workspace_words()
    return torch.zeros(n, dtype=torch.uint64, device=device or "cuda")


def launch_config(schedule="persistent", integrator=2, block_threads=0, blocks_per_sm=0, chunk=0):
    L = SlmLaunch()
    L.schedule = SCHEDULES[schedule] if isinstance(schedule, str) else int(schedule)
    L.integrator = int(integrator)
    L.block_threads = int(block_threads)
    L.blocks_per_sm = int(blocks_per_sm)
    L.chunk = int(chunk)
    return L


def integrate_fields(params, seeds, mask, uv, slc, slt, work, schedule="persistent",
                     integrator=2, block_threads=0, blocks_per_sm=0, stream=None,
                     order=None, item_steps=None, chunk=0):
    """Trace every seed's d*d jittered trajectories, adding into slc/slt (uint64).

    ``order`` (uint32 per seed, optional) issues seeds in that order (results
    unchanged); ``item_steps`` (uint16 per trajectory, optional) receives each
    trajectory's RK step count."""
    lib = _lib.load()
    nxy = params.nxy_padded
    _need(seeds, torch.float32, 2 * params.n_seed_points, "seeds")
    _need(mask, torch.uint8, nxy, "mask")
    _need(uv, torch.float32, 2 * nxy, "uv")
    _need(slc, torch.uint64, nxy, "slc")
    _need(slt, torch.uint64, nxy, "slt")
    _need(work, torch.uint64, lib.slm_fields_workspace_words(), "workspace")
    L = launch_config(schedule, integrator, block_threads, blocks_per_sm, chunk)
    if order is not None:
        _need(order, torch.uint32, int(params.n_seed_points), "order")
    if item_steps is not None:
        d = int(params.subpixel_seed_point_density)
        n_items = (int(params.n_seed_points) - int(params.seeds_chunk_offset)) * d * d
        _need(item_steps, torch.uint16, n_items, "item_steps")
    check(lib.slm_integrate_fields_scheduled(sref(params), sref(L), ptr(seeds), ptr(mask), ptr(uv),
                                             None, ptr(slc), ptr(slt), ptr(work), ptr(order),
                                             ptr(item_steps), _stream(stream)))


def integrate_fields_pair(params_down, params_up, seeds, mask, uv, slc, slt, work, integrator=2,
                          block_threads=0, blocks_per_sm=0, chunk=0, order=None, order_up=None,
                          stream=None):
    """Both directions in one persistent launch.  ``slc``/``slt``: uint64
    tensors of shape [2, nxy] (downstream, upstream; any stride between the
    two rows), each row as ``integrate_fields`` of that direction.  ``order``
    is the queue order of both directions unless ``order_up`` gives the
    upstream one."""
    lib = _lib.load()
    nxy = params_down.nxy_padded
    _need(seeds, torch.float32, 2 * params_down.n_seed_points, "seeds")
    _need(mask, torch.uint8, nxy, "mask")
    _need(uv, torch.float32, 2 * nxy, "uv")
    for name, t in (("slc", slc), ("slt", slt)):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.uint64 and t.dim() == 2
                and t.shape[0] == 2 and t.shape[1] >= nxy and t.stride(1) == 1):
            raise ValueError("{} must be a CUDA uint64 [2, nxy] tensor with contiguous rows".format(name))
    if slc.stride(0) != slt.stride(0):
        raise ValueError("slc and slt must have the same row stride")
    _need(work, torch.uint64, lib.slm_fields_workspace_words(), "workspace")
    if order is not None:
        _need(order, torch.uint32, int(params_down.n_seed_points), "order")
    if order_up is not None:
        _need(order_up, torch.uint32, int(params_down.n_seed_points), "order_up")
    L = launch_config("persistent", integrator, block_threads, blocks_per_sm, chunk)
    check(lib.slm_integrate_fields_pair(sref(params_down), sref(params_up), sref(L), ptr(seeds), ptr(mask),
                                        ptr(uv), ptr(slc), ptr(slt), int(slc.stride(0)), ptr(work), ptr(order),
                                        ptr(order_up), _stream(stream)))


def integrate_trajectory(params, n_chunk, seeds, mask, uv, traj, nsteps, length,
                         integrator=2, stream=None):
    """Record one trajectory per seed of the chunk starting at params.seeds_chunk_offset."""
    lib = _lib.load()
    nxy = params.nxy_padded
    _need(seeds, torch.float32, 2 * params.n_seed_points, "seeds")
    _need(mask, torch.uint8, nxy, "mask")
    _need(uv, torch.float32, 2 * nxy, "uv")
    _need(traj, torch.int8, 2 * n_chunk * params.max_n_steps, "trajectories")
    _need(nsteps, torch.uint16, n_chunk, "nsteps")
    _need(length, torch.float32, n_chunk, "length")
    check(lib.slm_integrate_trajectory(sref(params), int(integrator), int(n_chunk), ptr(seeds),
                                       ptr(mask), ptr(uv), None, ptr(traj), ptr(nsteps),
                                       ptr(length), _stream(stream)))


# ------------------------------------------------------------------ KDE
def histogram_univariate(params, data, hist, stream=None):
    _need(data, torch.float32, None, "data")
    _need(hist, torch.uint32, int(params.n_hist_bins), "histogram")
    check(_lib.load().slm_histogram_univariate(sref(params), ptr(data), int(data.numel()),
                                                ptr(hist), _stream(stream)))


def histogram_bivariate(params, data, hist, stream=None):
    _need(data, torch.float32, None, "data")
    nb = int(params.n_hist_bins)
    _need(hist, torch.uint32, nb * nb, "histogram")
    check(_lib.load().slm_histogram_bivariate(sref(params), ptr(data), int(data.numel() // 2),
                                               ptr(hist), _stream(stream)))


def pdf_univariate(params, hist, pdf, stream=None):
    _need(hist, torch.uint32, int(params.n_hist_bins), "histogram")
    _need(pdf, torch.float32, int(params.n_pdf_points), "pdf")
    check(_lib.load().slm_pdf_univariate(sref(params), ptr(hist), ptr(pdf), _stream(stream)))


def pdf_bivariate_rows(params, hist, partial, stream=None):
    nb = int(params.n_hist_bins)
    _need(hist, torch.uint32, nb * nb, "histogram")
    _need(partial, torch.float32, nb * nb, "partial pdf")
    check(_lib.load().slm_pdf_bivariate_rows(sref(params), ptr(hist), ptr(partial), _stream(stream)))


def pdf_bivariate_cols(params, partial, pdf, stream=None):
    nb, np_ = int(params.n_hist_bins), int(params.n_pdf_points)
    _need(partial, torch.float32, nb * nb, "partial pdf")
    _need(pdf, torch.float32, np_ * np_, "pdf")
    check(_lib.load().slm_pdf_bivariate_cols(sref(params), ptr(partial), ptr(pdf), _stream(stream)))
