"""The Mapping stage: passes 1 and 2 with the region's grids on the compute device.

What the passes compute (the reference's ``streamlines.mapping.Mapping``,
python/streamlines/mapping.py:235-560, computes the same arrays):

Pass 1 maps the whole region coarsely.  Inside the window around the
unmasked pixels it flags midslopes and ridges (from the sla angle), maps
channels and segments with the coarse thresholds, and keeps the segment
labels as the region's coarse subsegments.

Pass 2 revisits each coarse subsegment L, in ascending label order.  Its
pixels, grown by 2 pixels for a left flank (L < 0) or 1 for a right flank,
form the working region; the channel threshold comes from the KDE of that
region's downstream slt (clamped to [min, max], else the guess or half of
it); channels and segments are mapped there with the fine thresholds; the
hillslope length of every unmasked midslope pixel is traced along its
streamline to the channel; each fine subsegment's lengths give count / mean
/ standard deviation, and its mean is painted on its pixels.  Only the
subsegment's own (ungrown) pixels take the new lengths and flags back.

How this implementation is organised:

* ``_Roi`` holds the region's grids -- flags (uint32), coarse labels
  (int32), hillslope lengths (float32), the job's base mask, the
  downstream fields the mapping reads -- as tensors on one device, for both
  passes and every subsegment.
* ``_Window`` is an axis-aligned window of the region (a bounding box
  widened by the pad): crops, the Info of its kernels, and the write-back.
* An engine maps channels and segments in a window and traces the lengths:
  ``DeviceEngine`` keeps the window's grids on the GPU from the crop to the
  lengths (``DeviceMapping`` fed with device tensors);  ``WrapperEngine``
  runs the reference-shaped wrappers with a kernel runner (the oracle, to
  check the passes against the reference on the CPU).
* Region growing is a 3x3 max-pool per pixel of growth (binary dilation with
  the 8-neighbour structure), bounding boxes come from row / column
  reductions, and the write-back is a masked scatter, all on the device.
  The per-subsegment statistics, over the few midslope lengths, use pandas
  as the reference does, so the means painted are the reference's; the KDE's
  data selection runs on host copies of the window (the KDE itself runs on
  the GPU).

The hillslope lengths are measured as the reference's pass 2 measures
them, by fast marching (``hsl_method="fmm"``, the default): every labelled
subsegment of the window gets twice the mean eikonal distance of its grown
region from its thin channel (``slm_b200.fmm``, the CUDA kernel
``slm_fmm_lengths``), and each subsegment's value is painted on its pixels.
``hsl_method="traced"`` takes instead the lengths traced along streamlines
from the midslopes, the alternative the reference keeps beside it.  Pass 3
(scikit-image's rank filters, absent) is not built.
"""
from __future__ import annotations

import types

import numpy as np
import torch
import torch.nn.functional as F

from . import mapping as M
from .device import traced
from .useful import Info, default_parameters, vprint

MAPPING_PARAMETERS = dict(vars(default_parameters().mapping))
MAPPING_PARAMETERS.update(do_map_channels_segments=True, do_map_hsl=True, midslope_filter_sigma=5.0,
                          midslope_threshold=0.03, ridge_filter_sigma=2.0, ridge_threshold=0.8,
                          n_hsl_averaging_threshold=1, hsl_averaging_threshold=5.0)
# this project's: threads (each with its own CUDA stream) pass 2 runs its
# independent coarse subsegments on when the grids are on the GPU
MAPPING_PARAMETERS.update(pass2_workers=6)

HSL_COLUMNS = ("count", "mean [m]", "stddev [m]")
FMM_ORDER = 2  # skfmm.distance's default order, which the reference's call takes


# ------------------------------------------------------------------ grid helpers
def grow(region, n_pixels):
    """``region`` (bool [X, Y]) grown by ``n_pixels`` with the 8-neighbour
    structure; outside the grid counts as not in the region."""
    x = region.to(torch.float32)[None, None]
    for _ in range(int(n_pixels)):
        x = F.max_pool2d(x, 3, stride=1, padding=1)
    return x[0, 0] > 0


def label_boxes(grid, labels):
    """(x_min, x_max, y_min, y_max) of the pixels of each of ``labels`` (an
    ascending int array) in the int grid ``grid`` [X, Y]; a host int64 array
    [len(labels), 4].  A label with no pixel gets (X + Y, -1, X + Y, -1)."""
    dev = grid.device
    keys = torch.from_numpy(np.asarray(labels, dtype=np.int64)).to(dev)
    n, (X, Y) = keys.numel(), grid.shape
    out = torch.empty((4, n), dtype=torch.int64, device=dev)
    if n == 0:
        return out.t().cpu().numpy()
    flat = grid.reshape(-1).to(torch.int64)
    pos = torch.searchsorted(keys, flat).clamp_(max=n - 1)
    at = torch.nonzero(keys[pos] == flat).flatten()
    k = pos[at]
    xs, ys = at // Y, at % Y
    for row, v, how, init in ((0, xs, "amin", X + Y), (1, xs, "amax", -1), (2, ys, "amin", X + Y),
                              (3, ys, "amax", -1)):
        out[row].fill_(init).scatter_reduce_(0, k, v, how)
    return out.t().cpu().numpy()


def _paste(dst, dst_origin, src, src_origin):
    """Copy ``src`` into ``dst`` where they overlap; each array's origin is
    the grid position of its element (0, 0)."""
    lo = [max(d, s_) for d, s_ in zip(dst_origin, src_origin)]
    hi = [min(d + n, s_ + m) for d, n, s_, m in zip(dst_origin, dst.shape, src_origin, src.shape)]
    if lo[0] < hi[0] and lo[1] < hi[1]:
        dst[lo[0] - dst_origin[0]:hi[0] - dst_origin[0], lo[1] - dst_origin[1]:hi[1] - dst_origin[1]] = \
            src[lo[0] - src_origin[0]:hi[0] - src_origin[0], lo[1] - src_origin[1]:hi[1] - src_origin[1]]


def bounding_box(on):
    """(x_min, x_max, y_min, y_max) of the True pixels of ``on`` (bool [X, Y])."""
    xs = torch.nonzero(on.any(dim=1)).flatten()
    ys = torch.nonzero(on.any(dim=0)).flatten()
    if xs.numel() == 0:
        raise ValueError("no unmasked pixel to map")
    return int(xs[0]), int(xs[-1]), int(ys[0]), int(ys[-1])


class _Window:
    """The bounding box of ``on`` widened by ``pad`` on every side; ``origin``:
    the grid position of ``on``'s element (0, 0) when ``on`` is a crop."""

    def __init__(self, on, pad, origin=(0, 0)):
        x0, x1, y0, y1 = bounding_box(on)
        x0, x1, y0, y1 = x0 + origin[0], x1 + origin[0], y0 + origin[1], y1 + origin[1]
        self.pad = pad
        self.nx, self.ny = x1 + 1 - x0, y1 + 1 - y0  # the box itself
        self.box = (x0, x1, y0, y1)
        self.sl = (slice(x0 - pad, x1 + pad + 1), slice(y0 - pad, y1 + pad + 1))

    def info(self, stage, coarse_label=None):
        info = Info(stage.state, stage.trace, stage.geodata.roi_pixel_size, mapping=stage,
                    coarse_label=coarse_label)
        info.set_xy(self.nx, self.ny, self.pad)
        return info

    def of(self, t):
        return t[self.sl]


class _Roi:
    """The region's grids on one device."""

    def __init__(self, nxp, nyp, trace, uv, base_mask, device):
        dev = device
        self.device = dev
        self.mapping = torch.zeros((nxp, nyp), dtype=torch.int64, device=dev)  # uint32 flags held in int64
        self.coarse = torch.zeros((nxp, nyp), dtype=torch.int32, device=dev)
        self.hsl = torch.zeros((nxp, nyp), dtype=torch.float32, device=dev)
        self.base = torch.from_numpy(np.ascontiguousarray(base_mask)).to(dev)
        self.uv = torch.from_numpy(np.ascontiguousarray(uv, dtype=np.float32)).to(dev)
        self.slt = torch.from_numpy(np.ascontiguousarray(trace.slt_array, dtype=np.float32)).to(dev)
        self.slc = torch.from_numpy(np.ascontiguousarray(trace.slc_array, dtype=np.float64)).to(dev)
        self.sla_h = np.asarray(trace.sla_array)
        self.slt_h = np.asarray(trace.slt_array)
        self.uv_h = np.asarray(uv)


def _u32(t):
    """int64 flag tensor -> uint32 NumPy array."""
    return t.to(torch.int64).cpu().numpy().astype(np.uint32)


# ------------------------------------------------------------------ engines
class WrapperEngine:
    """The mapping sequence through the reference-shaped wrappers
    (mapping.map_channels_segments), each kernel through ``runner``."""

    def __init__(self, runner):
        self.runner = runner

    def map(self, info, win, roi, mask, mapping):
        """Channels and segments in the window; returns (ok, flags int64
        tensor, labels int32 tensor) on the region's device."""
        sl = win.sl
        data = types.SimpleNamespace(
            mask_array=np.ascontiguousarray(mask.cpu().numpy()), uv_array=np.ascontiguousarray(roi.uv_h[sl]),
            mapping_array=_u32(mapping), slt_array=np.ascontiguousarray(roi.slt_h[sl]),
            slc_array=np.ascontiguousarray(roi.slc[sl].cpu().numpy()), label_array=None,
            count_array=None, link_array=None, channel_label_array=None)
        ok = M.map_channels_segments(None, info, data, runner=self.runner)
        self.data = data
        lab = data.label_array if data.label_array is not None else np.zeros(mask.shape, np.int32)
        return (ok, torch.from_numpy(data.mapping_array.astype(np.int64)).to(roi.device),
                torch.from_numpy(np.ascontiguousarray(lab, dtype=np.int32)).to(roi.device))

    def fmm_lengths(self, info, flags, labels, selected, dx, order):
        """The fast-marching length (int32) of each ``selected`` fine label
        of the window, through the runner's ``fmm_solver`` when it has one
        (the oracle's), else the CUDA kernel."""
        from . import fmm
        return fmm.fmm_lengths(labels, flags, int(info.is_thinchannel), selected, dx, order,
                               solver=getattr(self.runner, "fmm_solver", None))

    def lengths(self, info, mapping, n):
        """The doubled hillslope lengths of the window's unmasked midslope
        pixels (row-major order), or None when there is none."""
        d = self.data
        d.mapping_array = _u32(mapping)
        d.subsegment_hsl_array = np.zeros(n, dtype=np.float32)
        if not M.hsl(None, info, d, False, runner=self.runner):
            return None
        return d.subsegment_hsl_array


class DeviceEngine:
    """The mapping sequence with the window's grids resident on the GPU
    (``mapping_device.DeviceMapping`` over device tensors).  ``status`` ORs
    the kernels' status words (1: a walk the reference leaves unbounded hit
    its cap; 2: a read the reference would make outside the grid was
    skipped), as ``mapping.DeviceRunner`` does."""

    def __init__(self, device=None):
        self.device = device
        self.status = 0

    def map(self, info, win, roi, mask, mapping):
        from .mapping_device import DeviceMapping
        sl = win.sl
        data = types.SimpleNamespace(mask_array=mask, uv_array=roi.uv[sl], mapping_array=mapping.to(torch.uint32),
                                     slt_array=roi.slt[sl], slc_array=roi.slc[sl])
        self.dm = DeviceMapping(info, data, device=roi.device)
        with torch.cuda.device(roi.device):
            ok = self.dm.map_channels_segments()
        self.status |= self.dm.status
        shape = mask.shape
        return (ok, self.dm.mapping.view(shape).to(torch.int64),
                self.dm.label.view(shape).view(torch.int32).clone())

    def fmm_lengths(self, info, flags, labels, selected, dx, order):
        from . import fmm
        with torch.cuda.device(labels.device):
            return fmm.fmm_lengths(labels, flags, int(info.is_thinchannel), selected, dx, order)

    def lengths(self, info, mapping, n):
        self.dm.mapping.copy_(mapping.reshape(-1).to(torch.uint32))
        if n == 0:
            return None
        with torch.cuda.device(self.dm.dev):
            return self.dm.hsl(False)


def subsegment_order(coarse, base, labels, boxes, pad):
    """The order constraints among pass 2's coarse subsegments: subsegment j
    reads the flags of its window (the box of its own pixels grown by 1 or 2
    px, within the frame, widened by ``pad``) and writes only its own
    unmasked pixels.  For every pair whose writes fall in the other's window
    the lower label goes first.  Returns (successor lists, predecessor
    counts), by position in ``labels``."""
    n = len(labels)
    index = {int(lab): i for i, lab in enumerate(labels)}
    nx, ny = coarse.shape
    written = np.where(base, 0, coarse)
    succ = [set() for _ in range(n)]
    for j in range(n):
        g = 2 if labels[j] < 0 else 1
        x0, x1, y0, y1 = (int(v) for v in boxes[j])
        x0, x1 = max(pad, x0 - g) - pad, min(nx - 1 - pad, x1 + g) + pad
        y0, y1 = max(pad, y0 - g) - pad, min(ny - 1 - pad, y1 + g) + pad
        for v in np.unique(written[max(0, x0):x1 + 1, max(0, y0):y1 + 1]):
            i = index.get(int(v))
            if i is None or i == j:
                continue
            a, b = (i, j) if i < j else (j, i)
            succ[a].add(b)
    indeg = [0] * n
    for a in range(n):
        for b in succ[a]:
            indeg[b] += 1
    return [sorted(x) for x in succ], indeg


# ------------------------------------------------------------------ subsegment statistics
def length_statistics(fine_labels, lengths, coarse_label):
    """Count, mean and standard deviation of the lengths of each nonzero
    fine label, one row per distinct label in ascending order, indexed by
    (fine, coarse) -- pandas' groupby statistics, as the reference's
    parse_hsl (mapping.py:920-944) takes them.  None when they cannot be
    formed."""
    import pandas as pd
    fine_labels = np.asarray(fine_labels, dtype=np.int32)
    lengths = np.asarray(lengths)  # float32 traced lengths, int32 fast-marching ones
    keep = fine_labels != 0
    try:
        rows = pd.Series(lengths[keep]).groupby(fine_labels[keep]).agg(["count", "mean", "std"])
    except Exception:  # noqa: BLE001 - a failed subsegment is skipped, as in the reference
        return None
    rows.columns = list(HSL_COLUMNS)
    coarse = np.full(len(rows), coarse_label, dtype=np.asarray(coarse_label).dtype)
    rows.index = pd.MultiIndex.from_arrays([rows.index.to_numpy(np.int32), coarse], names=["fine", "coarse"])
    return rows


_EMPTY_STATS = {}


def empty_statistics(coarse_label):
    """``length_statistics``' table with no rows (its columns, dtypes and
    index levels), made once per dtype of the coarse label."""
    key = np.asarray(coarse_label).dtype
    if key not in _EMPTY_STATS:
        _EMPTY_STATS[key] = length_statistics(np.array([1], np.int32), np.array([0], np.int32),
                                              coarse_label).iloc[0:0]
    return _EMPTY_STATS[key].copy()


def paint_means(labels, stats, min_count, device):
    """Each listed fine subsegment's mean length on its pixels (0 when it has
    fewer than ``min_count`` lengths, and on unlisted pixels); float32."""
    if stats is None or len(stats) == 0:
        return torch.zeros(labels.shape, dtype=torch.float32, device=device)
    fine = stats.index.get_level_values("fine").to_numpy(np.int64)
    value = np.where(stats["count"].to_numpy() >= min_count, stats["mean [m]"].to_numpy(), 0.0)
    return paint_values(labels, fine, value, device)


def paint_values(labels, fine, value, device):
    """``value[i]`` (rounded to float32) on the pixels labelled ``fine[i]``;
    0 elsewhere."""
    out = torch.zeros(labels.shape, dtype=torch.float32, device=device)
    fine = np.asarray(fine, dtype=np.int64)
    if fine.size == 0:
        return out
    order = np.argsort(fine, kind="stable")
    keys = torch.from_numpy(fine[order]).to(device)
    vals = torch.from_numpy(np.asarray(value)[order].astype(np.float32)).to(device)
    lab = labels.to(torch.int64)
    k = torch.searchsorted(keys, lab).clamp_(max=keys.numel() - 1)
    hit = keys[k] == lab
    out[hit] = vals[k[hit]]
    return out


# ------------------------------------------------------------------ the stage
class Mapping:
    """``state``: the job state (``reset_active_masks()``,
    ``merge_active_masks()``, ``add_active_mask()``, and the state
    parameters Info reads); ``imported_parameters``: the job's parameters
    (its 'mapping' section, or that section itself); ``geodata``:
    ``roi_nx``, ``roi_ny``, ``pad_width``, ``roi_pixel_size``;
    ``preprocess``: ``uv_array``; ``trace``: the trace parameters and
    ``slc_array`` / ``slt_array`` / ``sla_array``; ``analysis``: its
    ``estimate_channel_threshold`` (pass 2).

    ``runner``: a kernel runner (e.g. the oracle) -- the passes then run
    through the reference-shaped wrappers on the CPU; by default the grids
    live on the GPU (``device``) and the mapping sequence runs there.
    ``thin``: the one-pixel thinning of the midslope and ridge filters."""

    def __init__(self, state, imported_parameters, geodata, preprocess, trace, analysis=None, runner=None,
                 thin=None, device=None):
        params = dict(MAPPING_PARAMETERS)
        if imported_parameters:
            params.update(imported_parameters.get("mapping", imported_parameters))
        for k, v in params.items():
            setattr(self, k, v)
        self.state, self.geodata, self.preprocess, self.trace, self.analysis = \
            state, geodata, preprocess, trace, analysis
        self.thin = thin
        self.verbose = getattr(state, "verbose", False)
        if runner is not None and not isinstance(runner, M.DeviceRunner):
            self.engine, self.device = WrapperEngine(runner), torch.device("cpu")
        else:
            from .device import cuda_device
            self.device = device if device is not None else cuda_device(0, 0)
            self.engine = DeviceEngine(self.device)
        self._roi = None
        self.coarse_subsegments_list_array = np.zeros(0, np.int32)
        self.n_coarse_subsegments = 0
        self.hsl_mean_array = np.array([], dtype=np.float32)
        self.hsl_stats_df = None

    def print(self, *args, **kwargs):
        vprint(self.verbose, *args, **kwargs)

    # the region's grids as the reference keeps them: NumPy arrays
    @property
    def mapping_array(self):
        return _u32(self._roi.mapping)

    @property
    def coarse_subsegment_array(self):
        return self._roi.coarse.cpu().numpy()

    @property
    def merged_coarse_mask_array(self):
        return ~np.isin(self.coarse_subsegment_array, self.coarse_subsegments_list_array)

    @property
    def hsl_array(self):
        return self._roi.hsl.cpu().numpy()

    def _base_mask(self):
        self.state.reset_active_masks()
        return self.state.merge_active_masks()

    def _clear(self, flags):
        """Erase bits from every pixel of the region's flags."""
        self._roi.mapping &= ~int(flags)

    # ---------------------------------------------------------------- pass 1
    @traced("slm.Mapping.pass1")
    def pass1(self):
        self.print("\n**Pass#1 begin**")
        g = self.geodata
        pad = g.pad_width
        base = self._base_mask()
        roi = self._roi = _Roi(g.roi_nx + 2 * pad, g.roi_ny + 2 * pad, self.trace, self.preprocess.uv_array,
                               base, self.device)
        win = _Window(~roi.base, pad)
        info = win.info(self)
        info.set_thresholds(channel_threshold=self.coarse_channel_threshold,
                            segmentation_threshold=self.coarse_segmentation_threshold)
        # midslope and ridge flags from the sla angle (host filters) in a fresh window grid
        sl = win.sl
        filt = types.SimpleNamespace(mask_array=base[sl].copy(), sla_array=roi.sla_h[sl],
                                     mapping_array=np.zeros((win.nx + 2 * pad, win.ny + 2 * pad), np.uint32))
        M.map_midslopes(info, filt, self.midslope_filter_sigma, self.midslope_threshold, thin=self.thin)
        M.map_ridges(info, filt, self.ridge_filter_sigma, self.ridge_threshold, thin=self.thin)
        info.set_flags(self)
        flags = torch.from_numpy(filt.mapping_array.astype(np.int64)).to(roi.device)
        mask_w = win.of(roi.base)
        if self.do_map_channels_segments:
            ok, flags, labels = self.engine.map(info, win, roi, mask_w, flags)
            if not ok:
                self.print("A problem during mapping channels & segments")
            win.of(roi.mapping).copy_(flags)
            win.of(roi.coarse).copy_(labels)
            present = torch.unique(labels[~mask_w]).cpu().numpy()
            self.coarse_subsegments_list_array = np.sort(present[present != 0]).astype(np.int32)
            self.n_coarse_subsegments = int(self.coarse_subsegments_list_array.shape[0])
        elif not self.do_map_hsl:
            # the flags alone reach the region, on its unmasked pixels
            target = win.of(roi.mapping)
            target[~mask_w] |= flags[~mask_w]
        base = self._base_mask()
        if self.do_map_hsl:
            win = _Window(torch.from_numpy(~base).to(roi.device), pad)
            info = win.info(self)
            info.set_thresholds(segmentation_threshold=self.fine_segmentation_threshold)
        self.info = info
        self._clear(info.is_channelhead | info.is_thinchannel)
        self.print("**Pass#1 end**")

    # ---------------------------------------------------------------- pass 2
    @traced("slm.Mapping.pass2")
    def pass2(self, hsl_method="fmm"):
        """Per coarse subsegment (pass 1's labels, ascending): see the module
        docstring.  ``hsl_method``: "fmm" (the reference's measurement) or
        "traced".  Needs ``pass1`` and an ``analysis``."""
        import pandas as pd
        if hsl_method not in ("fmm", "traced"):
            raise ValueError("hsl_method {!r}: 'fmm' or 'traced'".format(hsl_method))
        if hsl_method == "traced" and self.do_measure_hsl_from_ridges:
            raise NotImplementedError("traced hillslope lengths start from the midslopes; the reference's "
                                      "traced measurement selects no seeds when measuring from ridges")
        self.print("\n**Pass#2 begin**")
        roi = self._roi
        pad = self.geodata.pad_width
        pixel_size = float(self.geodata.roi_pixel_size)
        quiet = getattr(self.state, "verbose", False)
        # the job's masks, without pass 1's mask of its coarse subsegments
        self.state.add_active_mask({"merged_coarse": self.merged_coarse_mask_array})
        frame = torch.ones_like(roi.base)
        frame[pad:-pad, pad:-pad] = False
        roi.hsl.zero_()
        # the job's masks do not change inside the loop
        base = torch.from_numpy(self._base_mask()).to(roi.device)
        coarse_labels = self.coarse_subsegments_list_array
        nxp, nyp = roi.coarse.shape
        boxes = label_boxes(roi.coarse, coarse_labels)

        def one(j, engine, analysis):
            """Coarse subsegment j; returns (mean, table) or None.  It writes
            the hillslope lengths and flags of its own unmasked pixels."""
            label = coarse_labels[j]
            x0, x1, y0, y1 = boxes[j]
            # the subsegment grown by 1 px (2 for a left flank), off the
            # frame, worked out on the crop its growth can reach
            g = 2 if label < 0 else 1
            cx, cy = max(0, int(x0) - g), max(0, int(y0) - g)
            crop = (slice(cx, min(nxp, int(x1) + g + 1)), slice(cy, min(nyp, int(y1) + g + 1)))
            region_c = grow(roi.coarse[crop] == int(label), g) & ~frame[crop]
            win = _Window(region_c, pad, origin=(cx, cy))
            info = win.info(self, coarse_label=label)
            region = torch.zeros((win.sl[0].stop - win.sl[0].start, win.sl[1].stop - win.sl[1].start),
                                 dtype=torch.bool, device=roi.device)
            _paste(region, (win.sl[0].start, win.sl[1].start), region_c, (cx, cy))
            mask_w = win.of(base) | ~region
            own_w = win.of(roi.coarse) == int(label)
            t = analysis.estimate_channel_threshold(types.SimpleNamespace(
                mask_array=mask_w.cpu().numpy(), slt_array=roi.slt_h[win.sl], sla_array=roi.sla_h[win.sl]),
                verbose=quiet)
            if t is None or t > self.max_channel_threshold:
                t = self.guess_channel_threshold
            elif t < self.min_channel_threshold:
                t = self.guess_channel_threshold / 2
            info.set_thresholds(channel_threshold=t, segmentation_threshold=self.fine_segmentation_threshold)
            ok, flags, labels = engine.map(info, win, roi, mask_w, win.of(roi.mapping).clone())
            if not ok:
                return None
            # this pass's channel heads are kept as WAS_CHANNELHEAD
            head = int(info.is_channelhead)
            flags = torch.where((flags & head) == head, flags | int(info.was_channelhead), flags)
            if hsl_method == "fmm":
                # every subsegment with an unmasked pixel, one length each:
                # its statistics row has count 1 and mean = the length, every
                # row is painted (no count threshold), and none passes the
                # count > 1 filter of the returned table
                fine = torch.unique(labels[~mask_w])
                fine = fine[fine != 0].cpu().numpy().astype(np.int32)
                lengths = engine.fmm_lengths(info, flags, labels, fine, pixel_size, FMM_ORDER)
                if not (lengths > 0).any():
                    return None
                painted = paint_values(labels, fine, lengths.astype(np.float64), roi.device)
                table = empty_statistics(label)
            else:
                picked = ((flags & int(info.is_midslope)) > 0) & ~mask_w
                fine = labels[picked].cpu().numpy()
                lengths = engine.lengths(info, flags, int(fine.shape[0]))
                if lengths is None:
                    return None
                stats = length_statistics(fine, np.asarray(lengths, dtype=np.float32), label)
                if stats is None or len(stats) == 0:
                    return None
                painted = paint_means(labels, stats, self.n_hsl_averaging_threshold, roi.device)
                table = stats[(stats["count"] > 1) & (stats["mean [m]"] > 5.0)]
            kept = painted[~torch.isnan(painted)]
            kept = kept[kept >= self.hsl_averaging_threshold].cpu().numpy()
            if kept.shape[0] == 0:
                return None
            # only the subsegment's own unmasked pixels take the results
            take = own_w & ~win.of(base)
            win.of(roi.hsl)[take] = torch.nan_to_num(painted, nan=0.0)[take]
            target = win.of(roi.mapping)
            target[take] |= flags[take]
            return np.mean(kept), table

        results = self._run_subsegments(one, roi, base, coarse_labels, boxes)
        means = [r[0] for r in results if r is not None]
        tables = [r[1] for r in results if r is not None]
        roi.hsl.nan_to_num_(nan=0.0)
        self.hsl_mean_array = np.array(means, dtype=np.float32) if means else np.array([], dtype=np.float32)
        self.hsl_stats_df = pd.concat(tables) if tables else None
        self.state.reset_active_masks()
        self.print("\n**Pass#2 end**")

    def _run_subsegments(self, one, roi, base, coarse_labels, boxes):
        """``one(j, engine, analysis)`` for every coarse subsegment j; the
        results in label order, identical to running them one after another
        in that order.  With the grids on the GPU they run on
        ``pass2_workers`` threads, each on its own CUDA stream with its own
        engine and analysis: subsegment j reads the flags in its window and
        writes flags and lengths only on its own unmasked pixels, so j waits
        for every lower-label subsegment with such pixels in its window, and
        a higher-label one with pixels in j's window waits for j."""
        import copy
        import heapq
        import threading
        from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
        n = len(coarse_labels)
        workers = int(getattr(self, "pass2_workers", 1)) if isinstance(self.engine, DeviceEngine) else 1
        if workers <= 1 or n <= 1:
            return [one(j, self.engine, self.analysis) for j in range(n)]
        succ, indeg = subsegment_order(roi.coarse.cpu().numpy(), base.cpu().numpy(), coarse_labels, boxes,
                                       self.geodata.pad_width)
        dev = roi.device
        torch.cuda.current_stream(dev).synchronize()
        local = threading.local()
        engines, lock, last_pdf = [], threading.Lock(), []

        def job(j):
            if not hasattr(local, "stream"):
                local.stream = torch.cuda.Stream(dev)
                local.engine = DeviceEngine(self.device)
                local.analysis = copy.copy(self.analysis)
                with lock:
                    engines.append(local.engine)
            with torch.cuda.device(dev), torch.cuda.stream(local.stream):
                r = one(j, local.engine, local.analysis)
                local.stream.synchronize()
            if j == n - 1 and hasattr(local.analysis, "mpdf_dslt"):
                last_pdf.append(local.analysis.mpdf_dslt)
            return r

        results = [None] * n
        ready = [j for j in range(n) if indeg[j] == 0]
        heapq.heapify(ready)
        with ThreadPoolExecutor(workers) as ex:
            running = {}
            while ready or running:
                while ready and len(running) < 2 * workers:
                    j = heapq.heappop(ready)
                    running[ex.submit(job, j)] = j
                done, _ = wait(running, return_when=FIRST_COMPLETED)
                for f in done:
                    j = running.pop(f)
                    results[j] = f.result()
                    for k in succ[j]:
                        indeg[k] -= 1
                        if indeg[k] == 0:
                            heapq.heappush(ready, k)
        for e in engines:
            self.engine.status |= e.status
        if last_pdf:  # the analysis ends with the last subsegment's pdf, as in order
            self.analysis.mpdf_dslt = last_pdf[0]
        return results

    def pass3(self):
        raise NotImplementedError("pass 3 smooths the hillslope lengths and the aspect with scikit-image's rank "
                                  "mean / median filters (mapping.py:562-1050), which are not available here")
