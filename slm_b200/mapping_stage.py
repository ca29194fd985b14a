"""The Mapping stage's first pass: coarse channels, subsegments, midslopes, ridges.

Mirrors ``streamlines.mapping.Mapping.pass1`` (python/streamlines/mapping.py:
235-345) over this package's mapping wrappers:

1. crop every grid to the bounding box of the merged active mask;
2. flag midslopes and ridges from the sla angle (``map_midslopes``,
   ``map_ridges``);
3. map channels and segments with the coarse thresholds
   (``map_channels_segments``);
4. record the coarse subsegment labels, the list of them, and the mask that
   selects them;
5. merge the flags back into the full ROI grid, then erase this pass's
   channel-head and thin-channel bits.

The per-subsegment hillslope-length helpers follow: ``select_subsegments``,
``measure_hsl_traced`` (the lengths kernel), ``parse_hsl`` (per-subsegment
statistics) and ``remap_hsl`` (mapping.py:819-976).

Kernels run through ``runner`` (default: the GPU, ``mapping.DeviceRunner``;
tests pass the oracle).  ``pass2`` runs the reference's second pass with the
hillslope lengths traced along streamlines, the alternative the reference
keeps beside its fast-marching measurement (skfmm, absent here).  The third
pass is not restated.
"""
from __future__ import annotations

import numpy as np

from . import mapping as M
from .useful import Data, Info, default_parameters, dilate, get_bbox, vprint

MAPPING_PARAMETERS = dict(vars(default_parameters().mapping))
MAPPING_PARAMETERS.update(do_map_channels_segments=True, do_map_hsl=True, midslope_filter_sigma=5.0,
                          midslope_threshold=0.03, ridge_filter_sigma=2.0, ridge_threshold=0.8,
                          n_hsl_averaging_threshold=1, hsl_averaging_threshold=5.0)


class Mapping:
    """``state``: the job state (``reset_active_masks()``,
    ``merge_active_masks()``, the state parameters Info reads);
    ``imported_parameters``: the job's parameters (its 'mapping' section, or
    that section itself); ``geodata``: ``roi_nx``, ``roi_ny``, ``pad_width``,
    ``roi_pixel_size``; ``preprocess``: ``uv_array``; ``trace``: the trace
    parameters and ``slc_array`` / ``slt_array`` / ``sla_array``."""

    def __init__(self, state, imported_parameters, geodata, preprocess, trace, analysis=None, runner=None,
                 thin=None):
        params = dict(MAPPING_PARAMETERS)
        if imported_parameters:
            params.update(imported_parameters.get("mapping", imported_parameters))
        for k, v in params.items():
            setattr(self, k, v)
        self.state, self.geodata, self.preprocess, self.trace, self.analysis = \
            state, geodata, preprocess, trace, analysis
        self.runner = runner
        self.thin = thin
        self.cl_state = None
        self.verbose = getattr(state, "verbose", False)
        self.vprogress = self.verbose

    def print(self, *args, **kwargs):
        vprint(self.verbose, *args, **kwargs)

    def _runner(self):
        if self.runner is None:
            self.runner = M.DeviceRunner()
        return self.runner

    def pass1(self):
        vprint(self.vprogress, "\n**Pass#1 begin**")
        pad = self.geodata.pad_width
        nxp = self.geodata.roi_nx + pad * 2
        nyp = self.geodata.roi_ny + pad * 2
        self.mapping_array = np.zeros((nxp, nyp), dtype=np.uint32)
        self.coarse_subsegment_array = np.zeros((nxp, nyp), dtype=np.int32)
        self.merged_coarse_mask_array = np.ones((nxp, nyp), dtype=bool)
        info = Info(self.state, self.trace, self.geodata.roi_pixel_size, mapping=self)
        self.state.reset_active_masks()
        mask_array = self.state.merge_active_masks()
        bbox, nxb, nyb = get_bbox(~mask_array)
        info.set_xy(nxb, nyb, pad)
        info.set_thresholds(channel_threshold=self.coarse_channel_threshold,
                            segmentation_threshold=self.coarse_segmentation_threshold)
        data = Data(info=info, bbox=bbox, pad=pad, mapping_array=self.mapping_array, mask_array=mask_array,
                    uv_array=self.preprocess.uv_array, slc_array=self.trace.slc_array,
                    slt_array=self.trace.slt_array, sla_array=self.trace.sla_array)
        M.map_midslopes(info, data, self.midslope_filter_sigma, self.midslope_threshold, thin=self.thin)
        M.map_ridges(info, data, self.ridge_filter_sigma, self.ridge_threshold, thin=self.thin)
        info.set_flags(self)
        if self.do_map_channels_segments:
            if not M.map_channels_segments(self.cl_state, info, data, verbose=self.verbose,
                                           runner=self._runner()):
                self.print("A problem during mapping channels & segments")
            self.mapping_array[data.bounds_grid] = data.mapping_array
            self.coarse_subsegment_array[data.bounds_grid] = data.label_array
            coarse = np.unique(data.label_array[~data.mask_array])
            self.coarse_subsegments_list_array = np.sort(coarse[coarse != 0])
            self.n_coarse_subsegments = self.coarse_subsegments_list_array.shape[0]
            for label in self.coarse_subsegments_list_array:
                self.merged_coarse_mask_array[self.coarse_subsegment_array == label] = False
        self.state.reset_active_masks()
        if self.do_map_hsl:
            del info, data
            mask_array = self.state.merge_active_masks()
            bbox, nxb, nyb = get_bbox(~mask_array)
            info = Info(self.state, self.trace, self.geodata.roi_pixel_size, mapping=self)
            info.set_xy(nxb, nyb, pad)
            info.set_thresholds(segmentation_threshold=self.fine_segmentation_threshold)
            data = Data(info=info, bbox=bbox, pad=pad, mapping_array=self.mapping_array, mask_array=mask_array)
        self.info = info
        bounds = data.bounds_grid
        self.mapping_array[bounds][~mask_array[bounds]] |= data.mapping_array[~mask_array[bounds]]
        self.mapping_array[(self.mapping_array & info.is_channelhead) != 0] ^= info.is_channelhead
        self.mapping_array[(self.mapping_array & info.is_thinchannel) != 0] ^= info.is_thinchannel
        vprint(self.vprogress, "**Pass#1 end**")

    # ---------------------------------------------- hillslope lengths of subsegments
    def select_subsegments(self, info, data, do_restrict=True):
        """mapping.py:819-839: the (fine) subsegment label of every unmasked
        midslope pixel (every unmasked pixel when not restricted), and the
        nonzero labels among them."""
        if do_restrict:
            if self.do_measure_hsl_from_ridges:
                pass  # the reference selects nothing new for ridges here
            else:
                sel = ((data.mapping_array & info.is_midslope) > 0) & (~data.mask_array)
                data.subsegment_label_array = data.label_array[sel].astype(np.int32)
        else:
            data.subsegment_label_array = data.label_array[~data.mask_array].astype(np.int32)
        unique = np.unique(data.subsegment_label_array)
        data.selected_subsegments_array = unique[unique != 0].astype(np.int32)
        self.n_subsegments = unique.size

    def measure_hsl_traced(self, info, data):
        """mapping.py:910-918: the hillslope length of every selected pixel,
        traced on the GPU (``slm_hillslope_lengths``)."""
        data.subsegment_hsl_array = np.zeros_like(data.subsegment_label_array, dtype=np.float32)
        return M.hsl(self.cl_state, info, data, self.do_measure_hsl_from_ridges, self.verbose,
                     runner=self._runner())

    def parse_hsl(self, info, data):
        """mapping.py:920-944: count, mean and standard deviation of the
        lengths per selected subsegment, as a DataFrame indexed by
        (fine, coarse) label."""
        import pandas as pd
        n = data.subsegment_hsl_array.shape[0]
        df = pd.DataFrame(np.zeros((n,), dtype=[("fine", np.int32), ("length", np.float32)]))
        df["fine"] = data.subsegment_label_array
        df["length"] = data.subsegment_hsl_array
        df = df[df.fine != 0]
        try:
            stats_df = pd.DataFrame(data.selected_subsegments_array, columns=["fine"])
            for stat, column in (("count", "count"), ("mean", "mean [m]"), ("std", "stddev [m]")):
                stats_df = stats_df.join(getattr(df.groupby("fine"), stat)(), on="fine")
                stats_df.rename(index=str, columns={"length": column}, inplace=True)
        except Exception:  # noqa: BLE001 - the reference reports failure, not the error
            self.print("Problem constructing HSL stats dataframe")
            return False
        stats_df["coarse"] = getattr(info, "coarse_label", None)
        stats_df.set_index(["fine", "coarse"], inplace=True)
        data.hsl_stats_df = stats_df
        return True

    def remap_hsl(self, info, data, n_hsl_averaging_threshold=None):
        """mapping.py:946-976: each subsegment's mean length painted on its
        pixels (0 where it has fewer than ``n_hsl_averaging_threshold``
        lengths); the mean of the painted values of at least
        ``hsl_averaging_threshold`` metres."""
        if n_hsl_averaging_threshold is None:
            n_hsl_averaging_threshold = self.n_hsl_averaging_threshold
        stats_df = data.hsl_stats_df
        try:
            data.hsl_array = np.zeros((info.nx_padded, info.ny_padded), dtype=np.float32)
            for idx, row in stats_df.iterrows():
                data.hsl_array[data.label_array == idx[0]] = (row["mean [m]"] if row["count"] >= n_hsl_averaging_threshold
                                                              else 0)
        except Exception:  # noqa: BLE001
            self.print("Problem with HSL stats dataframe")
            return False
        if stats_df.empty:
            return False
        hsl = data.hsl_array[~np.isnan(data.hsl_array)]
        hsl = hsl[hsl >= self.hsl_averaging_threshold]
        if hsl.shape[0] == 0:
            return False
        data.trace_mean_hsl = np.mean(hsl)
        return True

    def make_coarse_subsegment_masks(self, coarse_subsegment, is_left_or_right, raw_mask, dilated_mask):
        """mapping.py:348-386: the mask of one coarse subsegment (raw), and
        that dilated by 2 pixels for a left flank or 1 for a right flank,
        never into the pad; returns the dilated mask's bounding box."""
        raw_mask.fill(True)
        raw_mask[self.coarse_subsegment_array == coarse_subsegment] = False
        dilate(~raw_mask, n_iterations=(2 if is_left_or_right == "left" else 1), out=dilated_mask)
        np.invert(dilated_mask, out=dilated_mask)
        pad = self.geodata.pad_width
        dilated_mask[:pad, :] = True
        dilated_mask[:, :pad] = True
        dilated_mask[-pad:, :] = True
        dilated_mask[:, -pad:] = True
        return get_bbox(~dilated_mask)

    def pass2(self, hsl_method="traced"):
        """mapping.py:388-560, per coarse subsegment: its dilated mask and
        crop, the channel threshold from the crop's dslt pdf (clamped as
        ``mapping.subsegment_channel_threshold`` does), fine channels and
        segments, the hillslope lengths and their statistics, then the merge
        of the subsegment's lengths and flags into the ROI grids.

        The reference measures the lengths by fast marching (skfmm, absent
        here).  Its own alternative, kept in the same method but switched
        off, measures them along streamlines from the midslopes
        (``select_subsegments``, ``measure_hsl_traced``, ``parse_hsl``,
        ``remap_hsl``); that is the ``"traced"`` method, the only one here.
        Needs ``pass1`` and an ``analysis`` (``estimate_channel_threshold``)."""
        import pandas as pd
        if hsl_method != "traced":
            raise NotImplementedError("hsl_method {!r}: fast marching needs skfmm, which is not available "
                                      "here; use 'traced'".format(hsl_method))
        vprint(self.vprogress, "\n**Pass#2 begin**")
        self.vbackup = getattr(self.state, "verbose", False)
        pad = self.geodata.pad_width
        nxp = self.geodata.roi_nx + pad * 2
        nyp = self.geodata.roi_ny + pad * 2
        pixel_size = self.geodata.roi_pixel_size
        self.state.add_active_mask({"merged_coarse": self.merged_coarse_mask_array})
        raw_mask_array = np.zeros((nxp, nyp), dtype=bool)
        dilated_mask_array = np.zeros((nxp, nyp), dtype=bool)
        merged_mask_array = np.zeros((nxp, nyp), dtype=bool)
        self.hsl_array = np.zeros((nxp, nyp), dtype=np.float32)
        self.hsl_mean_array = np.array([], dtype=np.float32)
        self.hsl_stats_df = None
        for idx, coarse_subsegment in enumerate(self.coarse_subsegments_list_array):
            if idx > 0:
                merged_mask_array.fill(False)
            self.state.reset_active_masks()
            is_left_or_right = "left" if coarse_subsegment < 0 else "right"
            bbox, nxb, nyb = self.make_coarse_subsegment_masks(coarse_subsegment, is_left_or_right,
                                                               raw_mask_array, dilated_mask_array)
            info = Info(self.state, self.trace, pixel_size, mapping=self, coarse_label=coarse_subsegment)
            info.set_xy(nxb, nyb, pad)
            self.state.add_active_mask({"dilated_segment": dilated_mask_array})
            self.state.merge_active_masks(out=merged_mask_array)
            data = Data(info=info, bbox=bbox, pad=pad, mapping_array=self.mapping_array,
                        mask_array=merged_mask_array, uv_array=self.preprocess.uv_array,
                        slc_array=self.trace.slc_array, slt_array=self.trace.slt_array,
                        sla_array=self.trace.sla_array)
            t = self.analysis.estimate_channel_threshold(data, verbose=self.vbackup)
            if t is None or t > self.max_channel_threshold:
                t = self.guess_channel_threshold
            elif t < self.min_channel_threshold:
                t = self.guess_channel_threshold / 2
            data.channel_threshold = t
            info.set_thresholds(channel_threshold=data.channel_threshold,
                                segmentation_threshold=self.fine_segmentation_threshold)
            if not M.map_channels_segments(self.cl_state, info, data, verbose=self.verbose, runner=self._runner()):
                del data
                continue
            # this pass's channel heads are remembered as WAS_CHANNELHEAD
            data.mapping_array[(data.mapping_array & info.is_channelhead) == info.is_channelhead] \
                |= info.was_channelhead
            self.select_subsegments(info, data)
            if not self.measure_hsl_traced(info, data) or not self.parse_hsl(info, data) \
                    or not self.remap_hsl(info, data):
                del data
                continue
            self.hsl_mean_array = np.append(self.hsl_mean_array, data.trace_mean_hsl)
            keep = data.hsl_stats_df[(data.hsl_stats_df["count"] > 1) & (data.hsl_stats_df["mean [m]"] > 5.0)]
            self.hsl_stats_df = keep.copy() if self.hsl_stats_df is None else pd.concat([self.hsl_stats_df, keep])
            self.state.remove_active_mask("dilated_segment")
            self.state.add_active_mask({"raw_segment": raw_mask_array})
            self.state.merge_active_masks(out=merged_mask_array)
            bounds = data.bounds_grid
            data.hsl_array[np.isnan(data.hsl_array)] = 0.0
            self.hsl_array[bounds][~merged_mask_array[bounds]] = data.hsl_array[~merged_mask_array[bounds]]
            self.mapping_array[bounds][~merged_mask_array[bounds]] |= data.mapping_array[~merged_mask_array[bounds]]
            self.state.remove_active_mask("raw_segment")
            del data
        self.hsl_array[np.isnan(self.hsl_array)] = 0.0
        vprint(self.vprogress, "\n**Pass#2 end**")

    def pass3(self):
        raise NotImplementedError("pass 3 smooths the hillslope lengths and the aspect with scikit-image's rank "
                                  "mean / median filters (mapping.py:562-1050), which are not available here")
