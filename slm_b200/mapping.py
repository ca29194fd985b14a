"""Channel, segment and hillslope mapping: drop-ins for the reference's mapping
wrappers and the kernel sequence of ``Mapping.map_channels_segments``.

Each function mirrors one reference wrapper -- same signature
``fn(cl_state, info, data, verbose)``, same seed selection, same in-place
updates of ``data.mapping_array`` / ``count_array`` / ``link_array`` /
``label_array`` / ``channel_label_array`` / ``subsegment_hsl_array``, same
return value (``False``/``0`` on an empty seed list):

  connect_channel_pixels   connect.py:32-79        kernel connect_channels
  map_channel_heads        channelheads.py:33-80   kernel map_channel_heads
  prune_channel_heads      channelheads.py:82-118  kernel prune_channel_heads
  count_downchannels       countlink.py:36-81      kernel count_downchannels
  flag_downchannels        countlink.py:83-130     kernel flag_downchannels
  label_confluences        label.py:33-78          kernel label_confluences
  segment_channels         segment.py:34-93        kernel segment_downchannels
  segment_hillslopes       segment.py:95-146       kernel segment_hillslopes
  subsegment_flanks        segment.py:148-243      kernels subsegment_channel_edges,
                                                   subsegment_flanks, fix_right_flanks,
                                                   fix_left_flanks
  link_hillslopes          hillslopes.py:32-80     kernel hillslopes
  hsl                      lengths.py:33-92        kernel hillslope_lengths

``map_channels_segments`` follows mapping.py:627-677 (with the helpers
:695-775).  The host thinning step uses this project's Zhang-Suen thinning
(slm_b200.skeleton) in place of scikit-image's medial axis + skeletonize.

Kernels run through ``runner(name, params, seeds, arrays)``, which updates the
NumPy ``arrays`` (the reference kernel's buffers after ``seed_point``, in its
order) in place.  The default runner is the CUDA library (``DeviceRunner``).
Host relabelling keeps the reference's results where NumPy 2 would reject its
expressions: segment relabelling is a rank map (the reference's loop over
sorted labels gives the same values) and the left-flank sign fix-up is done in
64-bit arithmetic.
"""
from __future__ import annotations

import numpy as np

from .params import kernel_params
from .skeleton import zhang_suen
from .useful import pick_seeds, vprint


class DeviceRunner:
    """Runs one mapping kernel on the GPU: uploads the buffers, calls the C
    ABI entry point, copies the written buffers back into the arrays."""

    def __init__(self, device=None):
        self.device = device
        self.status = 0  # OR of the status words returned by the kernels
        self.seconds = {}  # wall time per kernel name (each call copies in and out)

    def __call__(self, name, params, seeds, arrays):
        import time
        from . import map_kernels
        t = time.perf_counter()
        st = map_kernels.run(name, params, seeds, arrays, self.device)
        self.seconds[name] = self.seconds.get(name, 0.0) + time.perf_counter() - t
        self.status |= st
        return st


_default_runner = None


def _runner(runner):
    global _default_runner
    if runner is not None:
        return runner
    if _default_runner is None:
        _default_runner = DeviceRunner()
    return _default_runner


def _u32(a):
    """uint32 view of a label array (the kernels treat int32 labels as uint)."""
    return a.view(np.uint32) if a.dtype == np.int32 else a


def _run(runner, kernel, info, seeds, arrays):
    info.n_seed_points = np.uint32(seeds.shape[0])
    prm = kernel_params(info, kernel.upper())
    return _runner(runner)(kernel, prm, seeds, arrays)


def connect_channel_pixels(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(map=data.mapping_array, flag=info.is_channel, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return None
    _run(runner, "connect_channels", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array])
    return True


def map_channel_heads(cl_state, info, data, verbose=False, runner=None):
    m = data.mapping_array
    m[(m & info.is_thinchannel) == info.is_thinchannel] |= info.is_channelhead
    seeds = pick_seeds(mask=data.mask_array, flag=info.is_channel, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "map_channel_heads", info, seeds, [data.mask_array, data.uv_array, m])
    return True


def prune_channel_heads(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array,
                       flag=info.is_channelhead, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return None
    _run(runner, "prune_channel_heads", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array])


def count_downchannels(cl_state, info, data, verbose=False, runner=None):
    m = data.mapping_array
    m[(m & info.is_thinchannel) != 0] ^= info.is_thinchannel
    seeds = pick_seeds(mask=data.mask_array, map=m, flag=info.is_channelhead, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "count_downchannels", info, seeds,
         [data.mask_array, data.uv_array, m, data.count_array, data.link_array])
    return True


def flag_downchannels(cl_state, info, data, verbose=False, do_reset_count=True, runner=None):
    m = data.mapping_array
    m[(m & info.is_thinchannel) != 0] ^= info.is_thinchannel
    if do_reset_count:
        data.count_array *= 0
    seeds = pick_seeds(mask=data.mask_array, map=m, flag=info.is_channelhead, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "flag_downchannels", info, seeds,
         [data.mask_array, data.uv_array, m, data.count_array, data.link_array])
    return True


def label_confluences(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array,
                       flag=info.is_thinchannel, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    dn_slt = np.ascontiguousarray(data.slt_array[:, :, 0], dtype=np.float32)
    _run(runner, "label_confluences", info, seeds,
         [data.mask_array, data.uv_array, dn_slt, data.mapping_array, data.count_array,
          data.link_array])
    return True


def segment_channels(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array,
                       flag=info.is_channelhead, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return 0
    _run(runner, "segment_downchannels", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array, data.count_array,
          data.link_array, _u32(data.label_array)])
    # relabel channel segments 1,2,3,... in label order (segment.py:83-88)
    lab = data.label_array
    pos = lab > 0
    labels = np.unique(lab[pos].ravel())
    if labels.size == 0:
        return 0
    lab[pos] = (np.searchsorted(labels, lab[pos]) + 1).astype(lab.dtype)
    return int(labels.size)


def link_hillslopes(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(mask=data.mask_array, map=~data.mapping_array,
                       flag=info.is_thinchannel, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "hillslopes", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array, data.count_array, data.link_array])
    return True


def segment_hillslopes(cl_state, info, data, verbose=False, runner=None):
    seeds = pick_seeds(mask=data.mask_array, map=~data.mapping_array,
                       flag=info.is_thinchannel, pad=info.pad_width)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "segment_hillslopes", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array, data.count_array,
          data.link_array, _u32(data.label_array)])
    return True


def subsegment_flanks(cl_state, info, data, verbose=False, runner=None):
    pad = info.pad_width
    arrays = [data.mask_array, data.uv_array, data.mapping_array, data.channel_label_array,
              data.link_array, _u32(data.label_array)]
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array,
                       flag=info.is_subsegmenthead, pad=pad)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "subsegment_channel_edges", info, seeds, arrays)
    flag = info.is_leftflank | info.is_thinchannel
    for kernel in ("subsegment_flanks", "fix_right_flanks"):
        seeds = pick_seeds(mask=data.mask_array, map=~data.mapping_array, flag=flag, pad=pad)
        if seeds.shape[0] == 0:
            return False
        _run(runner, kernel, info, seeds, arrays)
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array, flag=info.is_leftflank, pad=pad)
    if seeds.shape[0] == 0:
        return False
    _run(runner, "fix_left_flanks", info, seeds, arrays)
    return True


def hsl(cl_state, info, data, do_use_ridges, verbose=False, runner=None):
    flag = info.is_ridge if do_use_ridges else info.is_midslope
    seeds = pick_seeds(mask=data.mask_array, map=data.mapping_array, flag=flag, pad=info.pad_width)
    if seeds.shape[0] != data.subsegment_hsl_array.shape[0]:
        raise ValueError("Mismatched midslope/ridge point arrays: seed pts={0} traj len={1}"
                         .format(seeds.shape, data.subsegment_hsl_array.shape))
    if seeds.shape[0] == 0:
        return False
    _run(runner, "hillslope_lengths", info, seeds,
         [data.mask_array, data.uv_array, data.mapping_array, _u32(data.label_array),
          data.subsegment_hsl_array])
    if not do_use_ridges:
        data.subsegment_hsl_array *= 2.0
    return True


def fmm_lengths(cl_state, info, data, pixel_size, order=2, verbose=False, runner=None):
    """``Mapping.fmm_lengths`` (mapping.py:841-900) on ``data``: the
    fast-marching length of each of ``data.selected_subsegments_array`` from
    ``data.label_array`` and the thin-channel flags of
    ``data.mapping_array``, into ``data.subsegment_hsl_array`` (int32, as the
    reference's array is) and ``data.fmm_mean_hsl`` (the mean of the positive
    ones).  Returns False when none is positive.  The distances come from the
    runner's ``fmm_solver`` when it has one (the oracle's), else from the
    CUDA kernel ``slm_fmm_lengths`` on the runner's device."""
    from . import fmm
    r = _runner(runner)
    solver = getattr(r, "fmm_solver", None)
    label, flags = data.label_array, data.mapping_array
    if solver is None:
        import torch

        from .device import cuda_device
        dev = getattr(r, "device", None) or cuda_device(0, 0)
        label = torch.from_numpy(np.ascontiguousarray(label, dtype=np.int32)).to(dev)
        flags = torch.from_numpy(np.asarray(flags).astype(np.int64)).to(dev)
    hsl = fmm.fmm_lengths(label, flags, int(info.is_thinchannel), data.selected_subsegments_array,
                          float(pixel_size), order, solver=solver)
    data.subsegment_hsl_array = hsl
    positive = hsl[hsl > 0]
    if positive.size == 0:
        return False
    data.fmm_mean_hsl = np.mean(positive)
    vprint(verbose, "FMM mean HSL = {0:0.1f}m".format(data.fmm_mean_hsl))
    return True


# ------------------------------------------------------------------ sequence
def map_channels(info, data):
    """Channel pixels from the downstream fields (mapping.py:695-702)."""
    slt = data.slt_array[:, :, 0]
    slc = data.slc_array[:, :, 0]
    data.mapping_array[(slt >= info.channel_threshold) & (slt * 2 >= slc)] = info.is_channel


def thin_channels(info, data, device=None):
    """Thin channel + inter-channel pixels to a skeleton (mapping.py:707-719);
    on the GPU (``slm_thin``) when ``device`` is given, with the same result."""
    m = data.mapping_array
    channel = (((m & info.is_channel) == info.is_channel)
               | ((m & info.is_interchannel) == info.is_interchannel))
    if device is not None:
        from .skeleton import zhang_suen_device
        thin = zhang_suen_device(channel, device=None if device is True else device)
    else:
        thin = zhang_suen(channel)
    m[thin] |= info.is_thinchannel


def map_channels_segments(cl_state, info, data, do_map_channels_from_scratch=True,
                          do_map_segments=True, verbose=False, runner=None):
    """The kernel sequence of mapping.py:627-677 (with :695-775)."""
    nxp, nyp = data.mask_array.shape
    if do_map_channels_from_scratch:
        map_channels(info, data)
    if not connect_channel_pixels(cl_state, info, data, verbose, runner):
        return False
    r = _runner(runner)
    thin_channels(info, data, device=(r.device or True) if isinstance(r, DeviceRunner) else None)
    if not map_channel_heads(cl_state, info, data, verbose, runner):
        return False
    data.count_array = np.zeros((nxp, nyp), dtype=np.uint32)
    data.link_array = np.zeros((nxp, nyp), dtype=np.uint32)
    if not count_downchannels(cl_state, info, data, verbose, runner):
        return False
    if not flag_downchannels(cl_state, info, data, verbose, runner=runner):
        return False
    if not do_map_segments:
        return True
    if (not label_confluences(cl_state, info, data, verbose, runner)
            or not flag_downchannels(cl_state, info, data, verbose, runner=runner)
            or not flag_downchannels(cl_state, info, data, verbose, do_reset_count=False, runner=runner)
            or not flag_downchannels(cl_state, info, data, verbose, do_reset_count=False, runner=runner)):
        return False
    data.label_array = np.zeros((nxp, nyp), dtype=np.int32)
    if segment_channels(cl_state, info, data, verbose, runner) == 0:
        return False
    data.channel_label_array = data.label_array.copy().astype(np.uint32)
    if not link_hillslopes(cl_state, info, data, verbose, runner):
        return False
    if not segment_hillslopes(cl_state, info, data, verbose, runner):
        return False
    if not subsegment_flanks(cl_state, info, data, verbose, runner):
        return False
    lab = data.label_array
    neg = lab < 0
    lab[neg] = (-(lab[neg].astype(np.int64) + int(info.left_flank_addition))).astype(np.int32)
    vprint(verbose, "mapped channels and segments")
    return True


MAPPING_THRESHOLD_DEFAULTS = {"min_channel_threshold": 10, "guess_channel_threshold": 150,
                              "max_channel_threshold": 1000, "fine_segmentation_threshold": 10}


def subsegment_channel_threshold(data, mapping_params=None, analysis_params=None, pixel_size=None):
    """The channel threshold the reference's per-subsegment pass maps with
    (mapping.py:460-477): the KDE estimate on the dslt pdf
    (``analysis.estimate_channel_threshold``), replaced by the guess when
    there is none or it lies above the maximum, and by half the guess below
    the minimum.  Sets ``data.channel_threshold`` and returns it."""
    from .analysis import estimate_channel_threshold
    p = dict(MAPPING_THRESHOLD_DEFAULTS)
    p.update(mapping_params or {})
    t = estimate_channel_threshold(data, analysis_params, pixel_size)
    if t is None or t > p["max_channel_threshold"]:
        t = p["guess_channel_threshold"]
    elif t < p["min_channel_threshold"]:
        t = p["guess_channel_threshold"] / 2
    data.channel_threshold = t
    return t


def _thin_default(image):
    from .skeleton import zhang_suen_device
    return zhang_suen_device(image)


def map_midslopes(info, data, midslope_filter_sigma=5.0, midslope_threshold=0.03, thin=None):
    """Mapping.map_midslopes (mapping.py:778-791): unmasked pixels where the
    Gaussian-smoothed angle between the downstream and upstream sla departs
    from pi/4 by at most ``midslope_threshold``, thinned to one pixel, get
    IS_MIDSLOPE.  The reference thins with scikit-image's skeletonize; here
    ``thin`` (default: this package's Zhang-Suen thinning on the GPU) stands
    in, so which pixels the thinning keeps is not pinned to the reference."""
    from scipy.ndimage import gaussian_filter
    thin = thin or _thin_default
    dsla, usla = data.sla_array[:, :, 0], data.sla_array[:, :, 1]
    mid = np.zeros((info.nx_padded, info.ny_padded), dtype=bool)
    mid[(~data.mask_array) & (np.fabs(gaussian_filter((np.arctan2(dsla, usla) - np.pi / 4),
                                                      midslope_filter_sigma)) <= midslope_threshold)] = True
    data.mapping_array[thin(mid)] |= info.is_midslope


def map_ridges(info, data, ridge_filter_sigma=2.0, ridge_threshold=0.8, thin=None):
    """Mapping.map_ridges (mapping.py:793-816): unmasked pixels whose smoothed
    sla angle lies at least (pi/4) * ridge_threshold below pi/4, dilated twice
    with the 8-neighbour structure, holes filled, thinned to one pixel (the
    stand-in for skeletonize as in ``map_midslopes``), get IS_RIDGE."""
    from scipy.ndimage import binary_dilation, binary_fill_holes, gaussian_filter, generate_binary_structure
    thin = thin or _thin_default
    dsla, usla = data.sla_array[:, :, 0], data.sla_array[:, :, 1]
    nxp, nyp = info.nx_padded, info.ny_padded
    ridge = np.zeros((nxp, nyp), dtype=bool)
    fat = np.zeros((nxp, nyp), dtype=bool)
    ridge[(~data.mask_array) & ((gaussian_filter((np.arctan2(dsla, usla) - np.pi / 4), ridge_filter_sigma))
                                <= -(np.pi / 4) * ridge_threshold)] = True
    binary_dilation(ridge, structure=generate_binary_structure(2, 2), iterations=2, output=fat)
    binary_fill_holes(fat, output=fat)
    data.mapping_array[thin(fat)] |= info.is_ridge
