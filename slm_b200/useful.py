"""Parameter container, seed lists and trajectory statistics.

Mirrors the parts of the reference's ``python/streamlines/useful.py`` that the
trace, fields, mapping and KDE stages use: ``Data`` (:37-115), ``Info``
(:117-269), ``get_bbox`` (:271-290), ``create_seeds`` (:470-517),
``pick_seeds`` (:519-538) and ``compute_stats`` (:540-571).  Same attribute
names and derivations, so a caller of the reference's stage wrappers can pass
the same objects.  NumPy-2 spellings replace the removed aliases
(``np.bool8`` -> ``np.bool_``).
"""
from __future__ import annotations

import sys
from types import SimpleNamespace

import numpy as np

__all__ = ["Data", "Info", "get_bbox", "create_seeds", "pick_seeds", "compute_stats",
           "vprint", "default_parameters"]

# Flag bit order of Info.set_flags (reference useful.py:238-268): bit i = 2**i.
FLAG_NAMES = [
    "is_channel", "is_thinchannel", "is_interchannel", "is_channelhead",
    "is_channeltail", "is_majorconfluence", "is_minorconfluence", "is_majorinflow",
    "is_minorinflow", "is_leftflank", "is_rightflank", "is_midslope", "is_ridge",
    "was_channelhead", "is_subsegmenthead", "is_loop", "is_blockage",
]


def default_parameters():
    """The reference's default job parameters for the hot-path stages.

    Values of ``json/defaults.json`` sections ``state`` (:2-14), ``trace``
    (:60-76), ``analysis`` KDE keys (:86-101) and ``mapping`` (:137-170) that the
    trace, fields, mapping and KDE stages read.
    """
    state = SimpleNamespace(verbose=False, gpu_verbose=False, debug=False,
                            cl_platform=0, cl_device=0, gpu_memory_limit_pc=90,
                            n_work_items=32, chunk_size_factor=20,
                            max_time_per_kernel=5.0)
    trace = SimpleNamespace(subpixel_seed_point_density=3, jitter_magnitude=1.0,
                            n_trajectory_seed_points=1000, do_shuffle_seed_points=True,
                            shuffle_rng_seed=1, max_length=1000.0,
                            interchannel_max_n_steps=5, integration_halt_threshold=0.01,
                            trajectory_resolution=128, integrator_step_factor=0.5,
                            max_integration_step_error=0.03, do_trace_upstream=True,
                            do_trace_downstream=True)
    analysis = SimpleNamespace(n_hist_bins=2048, n_pdf_points=256,
                               marginal_distbn_kde_bandwidth=10.0,
                               joint_distbn_kde_bandwidth=5.0,
                               marginal_distbn_kde_kernel="epanechnikov",
                               joint_distbn_kde_kernel="gaussian")
    mapping = SimpleNamespace(do_measure_hsl_from_ridges=False,
                              coarse_segmentation_threshold=1000,
                              coarse_channel_threshold=1000,
                              fine_segmentation_threshold=10,
                              min_channel_threshold=10, guess_channel_threshold=150,
                              max_channel_threshold=1000)
    return SimpleNamespace(state=state, trace=trace, analysis=analysis, mapping=mapping)


class Data:
    """Arrays handed between stages, cropped to ``bbox`` widened by ``pad``.

    Reference ``useful.py:37-115``.
    """

    def __init__(self, info=None, bbox=None, pad=0, mask_array=None, uv_array=None,
                 mapping_array=None, traj_stats_df=None, sla_array=None,
                 slc_array=None, slt_array=None, hsl_array=None):
        if bbox is not None:
            bbox = [bbox[0] - pad, bbox[1] + pad, bbox[2] - pad, bbox[3] + pad]
            bounds_grid = np.index_exp[bbox[0]:(bbox[1] + 1), bbox[2]:(bbox[3] + 1)]
            bounds_slx = np.index_exp[bbox[0]:(bbox[1] + 1), bbox[2]:(bbox[3] + 1), :]
        else:
            bounds_grid = np.index_exp[:, :]
            bounds_slx = np.index_exp[:, :, :]
        # copies, as the reference takes them (large ones on several threads;
        # the grids the tracer uploads into page-locked memory)
        from .device import host_copy
        self.mask_array = host_copy(mask_array[bounds_grid], pinned=True)
        if mapping_array is not None:
            self.mapping_array = host_copy(mapping_array[bounds_grid])
        else:
            self.mapping_array = None
        self.uv_array = host_copy(uv_array[bounds_slx], pinned=True) if uv_array is not None else None
        self.sla_array = host_copy(sla_array[bounds_slx]) if sla_array is not None else None
        self.slc_array = host_copy(slc_array[bounds_slx]) if slc_array is not None else None
        self.slt_array = host_copy(slt_array[bounds_slx]) if slt_array is not None else None
        self.traj_stats_df = traj_stats_df
        self.bounds_grid = bounds_grid
        self.bounds_slx = bounds_slx
        self.count_array = None
        self.link_array = None
        self.label_array = None
        self.channel_label_array = None
        self.selected_subsegments_array = None
        self.traj_label_array = None
        self.traj_length_array = None
        self.subsegment_label_array = None
        self.subsegment_hsl_array = None
        self.hsl_array = host_copy(hsl_array[bounds_slx]) if hsl_array is not None else None


class Info:
    """Derived kernel parameters (reference ``useful.py:117-269``).

    ``state``, ``trace`` and ``mapping`` are objects carrying the job
    parameters of the same names as the reference's JSON sections.
    """

    def __init__(self, state, trace, pixel_size, mapping=None, n_seed_points=None,
                 coarse_label=None):
        self.state = state
        self.trace = trace
        self.mapping = mapping
        if mapping is not None:
            self.do_measure_hsl_from_ridges = mapping.do_measure_hsl_from_ridges
        else:
            self.do_measure_hsl_from_ridges = False
        self.segmentation_threshold = np.uint32(0)
        self.channel_threshold = np.uint32(0)
        if coarse_label is not None:
            self.coarse_label = coarse_label
        if trace.max_length == np.float32(0.0):
            max_length = np.finfo(np.float32).max
        else:
            max_length = trace.max_length
        max_n_steps = np.uint32(trace.max_length / trace.integrator_step_factor)
        if trace.interchannel_max_n_steps == 0:
            interchannel_max_n_steps = max_n_steps
        else:
            interchannel_max_n_steps = trace.interchannel_max_n_steps
        self.max_n_steps = np.uint32(max_n_steps)

        seed_point_density = np.float32(trace.subpixel_seed_point_density)
        subpixel_seed_span = 1 - 1.0 / seed_point_density
        subpixel_seed_step = subpixel_seed_span / max(seed_point_density, 1.0)

        self.debug = np.bool_(state.debug)
        self.verbose = np.bool_(state.gpu_verbose)
        self.n_trajectory_seed_points = np.uint32(trace.n_trajectory_seed_points)
        self.n_seed_points = np.uint32(0)
        self.n_padded_seed_points = np.uint32(0)
        self.do_shuffle = np.bool_(trace.do_shuffle_seed_points)
        self.shuffle_rng_seed = np.uint32(trace.shuffle_rng_seed)
        self.downup_sign = np.float32(np.nan)
        self.gpu_memory_limit_pc = np.uint32(state.gpu_memory_limit_pc)
        self.n_work_items = np.uint32(state.n_work_items)
        self.chunk_size_factor = np.uint32(state.chunk_size_factor)
        self.max_time_per_kernel = np.float32(state.max_time_per_kernel)
        self.integrator_step_factor = np.float32(trace.integrator_step_factor)
        self.max_integration_step_error = np.float32(trace.max_integration_step_error)
        self.adjusted_max_error = 0.85 * np.sqrt(trace.max_integration_step_error)
        self.integration_halt_threshold = np.float32(trace.integration_halt_threshold)
        self.max_length = np.float32(max_length / pixel_size)
        self.pixel_size = np.float32(pixel_size)
        self.trajectory_resolution = np.uint32(trace.trajectory_resolution)
        self.seeds_chunk_offset = np.uint32(0)
        self.subpixel_seed_point_density = np.uint32(trace.subpixel_seed_point_density)
        self.subpixel_seed_halfspan = np.float32(subpixel_seed_span / 2.0)
        self.subpixel_seed_step = np.float32(subpixel_seed_step)
        self.jitter_magnitude = np.float32(trace.jitter_magnitude)
        self.interchannel_max_n_steps = np.uint32(interchannel_max_n_steps)
        self.left_flank_addition = 2147483648
        self.set_flags(self)

    def set_xy(self, nx, ny, pad, bbox=None):
        self.bbox = bbox
        self.pad_width = pad
        self.nx = nx
        self.ny = ny
        self.nx_padded = self.nx + self.pad_width * 2
        self.ny_padded = self.ny + self.pad_width * 2

    def set_thresholds(self, segmentation_threshold=None, channel_threshold=None):
        if segmentation_threshold is not None:
            self.segmentation_threshold = segmentation_threshold
        if channel_threshold is not None:
            self.channel_threshold = channel_threshold

    def set_flags(self, obj):
        for idx, flag in enumerate(FLAG_NAMES):
            setattr(obj, flag, np.uint(2 ** idx))


def get_bbox(array):
    """Bounding box of the True pixels: ((x_min,x_max,y_min,y_max), nx, ny)."""
    cols = np.any(array, axis=0)
    rows = np.any(array, axis=1)
    x_min, x_max = np.where(rows)[0][[0, -1]]
    y_min, y_max = np.where(cols)[0][[0, -1]]
    return (x_min, x_max, y_min, y_max), (x_max + 1 - x_min), (y_max + 1 - y_min)


def dilate(array, n_iterations=1, out=None):
    """Binary dilation with the 8-neighbour structure (useful.py:573-591)."""
    from scipy.ndimage import binary_dilation, generate_binary_structure
    return binary_dilation(array, structure=generate_binary_structure(2, 2), iterations=n_iterations, output=out)


def vprint(verbose, *args, **kwargs):
    if verbose:
        print(*args, **kwargs, flush=True)
        sys.stdout.flush()




def _shuffled_seeds(mask, pad, do_shuffle, rng_seed):
    """argwhere(~mask) - pad, shuffled as the reference shuffles it
    (useful.py:496-501), by ``slm_create_seeds`` (native host code: NumPy's
    legacy MT19937 Fisher-Yates shuffle with the swap partners drawn ahead).
    NumPy's global generator is left in the state the reference's shuffle
    leaves it in."""
    import ctypes

    from . import _lib
    m = np.ascontiguousarray(mask)
    if m.ndim != 2:
        raise ValueError("mask must be 2-D")
    m8 = m.view(np.uint8) if m.dtype == np.bool_ else (m != 0).view(np.uint8)
    L = _lib.load()
    n = ctypes.c_uint64(0)
    _lib.check(L.slm_create_seeds(m8.ctypes.data, m.shape[0], m.shape[1], int(pad), 0, 0, None, 0,
                                  ctypes.byref(n), None))
    if n.value == 0:
        if do_shuffle:
            np.random.seed(rng_seed)  # the shuffle of an empty list draws nothing
        return np.empty((0, 2), np.float32)
    out = np.empty((int(n.value), 2), np.float32)
    state = np.empty(625, np.uint32)
    _lib.check(L.slm_create_seeds(m8.ctypes.data, m.shape[0], m.shape[1], int(pad), 1 if do_shuffle else 0,
                                  int(rng_seed) & 0xFFFFFFFF, out.ctypes.data, out.shape[0],
                                  ctypes.byref(n), state.ctypes.data))
    if do_shuffle:
        np.random.set_state(("MT19937", state[:624].copy(), int(state[624]), 0, 0.0))
    return out


def create_seeds(mask, pad, n_work_items, n_seed_points=None, do_shuffle=True,
                 rng_seed=1, verbose=False):
    """Seed coordinates of the unmasked pixels (unpadded frame), optionally shuffled.

    The shuffle is NumPy's legacy ``RandomState`` stream seeded with
    ``rng_seed``, as in the reference (useful.py:496-501); the order fixes each
    seed's index and hence its jitter RNG stream.
    Returns ``(seed_point_array, n_seed_points, n_padded_seed_points)``.
    """
    vprint(verbose, "Generating seed points...", end="")
    seed_point_array = _shuffled_seeds(mask, pad, do_shuffle, rng_seed)
    if n_seed_points is not None and n_seed_points > 0:
        seed_point_array = seed_point_array[:n_seed_points].astype(np.float32)
    else:
        n_seed_points = seed_point_array.shape[0]
    pad_length = (np.uint32(np.round(n_seed_points / n_work_items + 0.5)) * n_work_items
                  - n_seed_points)
    n_padded_seed_points = n_seed_points + pad_length
    vprint(verbose, "done")
    return seed_point_array, n_seed_points, n_padded_seed_points  # a fresh array either way


def create_seeds_device(mask, pad, n_work_items, device, n_seed_points=None, do_shuffle=True, rng_seed=1,
                        verbose=False, mask_d=None, stream=None):
    """``create_seeds`` with the list built in device memory
    (``slm_create_seeds_device``): the same rows in the same order, and
    NumPy's global generator left where the reference's shuffle leaves it.

    ``mask``: the host mask (its shape gives the grid); ``mask_d``: the same
    mask already on ``device`` as uint8 (else it is uploaded).  Returns
    ``(seeds [n][2] float32 CUDA tensor, n_seed_points, n_padded_seed_points)``
    with ``n_seed_points`` rows (the first rows when truncated)."""
    seeds, n, npad, state = create_seeds_device_state(mask, pad, n_work_items, device, n_seed_points, do_shuffle,
                                                      rng_seed, verbose, mask_d, stream)
    if state is not None:
        np.random.set_state(state)
    return seeds, n, npad


def create_seeds_device_state(mask, pad, n_work_items, device, n_seed_points=None, do_shuffle=True, rng_seed=1,
                              verbose=False, mask_d=None, stream=None):
    """``create_seeds_device`` without touching NumPy's global generator: the
    generator state the reference's shuffle leaves (for
    ``numpy.random.set_state``; None without a shuffle) is returned as a
    fourth value instead, so the list can be built on another thread and the
    state applied where the reference's shuffle would run."""
    import ctypes

    import torch

    from . import _lib
    vprint(verbose, "Generating seed points on the GPU...", end="")
    nxp, nyp = mask.shape
    n_px = int(nxp) * int(nyp)
    if mask_d is None:
        m = np.ascontiguousarray(mask)
        m = m.view(np.uint8) if m.dtype == np.bool_ else (m != 0).view(np.uint8)
        mask_d = torch.from_numpy(m).to(device)
    L = _lib.load()
    ws = torch.empty(int(L.slm_create_seeds_device_workspace(n_px)), dtype=torch.uint8, device=device)
    out = torch.empty((max(1, n_px), 2), dtype=torch.float32, device=device)
    n = ctypes.c_uint64(0)
    state = np.empty(625, np.uint32)
    s = stream if stream is not None else torch.cuda.current_stream(device)
    _lib.check(L.slm_create_seeds_device(_lib.ptr(mask_d), int(nxp), int(nyp), int(pad), 1 if do_shuffle else 0,
                                         int(rng_seed) & 0xFFFFFFFF, _lib.ptr(out), out.shape[0], ctypes.byref(n),
                                         state.ctypes.data, _lib.ptr(ws), ws.numel(),
                                         ctypes.c_void_p(s.cuda_stream)))
    gen_state = ("MT19937", state[:624].copy(), int(state[624]), 0, 0.0) if do_shuffle else None
    n_all = int(n.value)
    rows = n_all
    if n_seed_points is not None and n_seed_points > 0:
        rows = min(int(n_seed_points), n_all)  # the count stays as asked, as create_seeds keeps it
    else:
        n_seed_points = n_all
    pad_length = (np.uint32(np.round(n_seed_points / n_work_items + 0.5)) * n_work_items
                  - n_seed_points)
    vprint(verbose, "done")
    return out[:rows], n_seed_points, n_seed_points + pad_length, gen_state


def pick_seeds(mask=None, map=None, flag=None, pad=None):
    """Seed coordinates of pixels selected by mask and/or mapping flag (useful.py:519-538)."""
    if mask is None and map is not None:
        seed_point_array = (np.argwhere((map & flag) > 0).astype(np.float32) - pad)
    elif mask is not None and map is None:
        seed_point_array = (np.argwhere(~mask).astype(np.float32) - pad)
    else:
        seed_point_array = (np.argwhere(~mask & ((map & flag) > 0)).astype(np.float32) - pad)
    return seed_point_array.copy()


def compute_stats(traj_length_array, traj_nsteps_array, pixel_size, verbose=False):
    """min/mean/max of length, step count and spacing per direction (useful.py:540-571).

    Returns a pandas DataFrame indexed like the reference's ``traj_stats_df``.
    """
    import pandas as pd
    lnds_stats = []
    for downup_idx in [0, 1]:
        ln = np.stack((traj_length_array[:, downup_idx] * pixel_size,
                       traj_nsteps_array[:, downup_idx])).T
        with np.errstate(divide="ignore", invalid="ignore"):
            lnds = np.column_stack((ln[:, 0], ln[:, 1], ln[:, 0] / ln[:, 1]))
        lnds_stats += [np.min(lnds, axis=0), np.mean(lnds, axis=0), np.max(lnds, axis=0)]
    lnds_stats_array = np.array(lnds_stats, dtype=np.float32)
    lnds_indexes = [np.array(["downstream"] * 3 + ["upstream"] * 3),
                    np.array(["min", "mean", "max", "min", "mean", "max"])]
    df = pd.DataFrame(data=lnds_stats_array, columns=["l", "n", "ds"], index=lnds_indexes)
    vprint(verbose, df.T)
    return df
