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
tests pass the oracle).  The reference's second pass measures hillslope
lengths by fast marching (skfmm), which is not available here.  That pass
and the third are not restated.
"""
from __future__ import annotations

import numpy as np

from . import mapping as M
from .useful import Data, Info, default_parameters, get_bbox, vprint

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

    def pass2(self):
        raise NotImplementedError("pass 2 measures hillslope lengths by fast marching (skfmm, mapping.py:388-560), "
                                  "which is not available here")

    def pass3(self):
        raise NotImplementedError("pass 3 filters pass 2's hillslope lengths (mapping.py:562-625)")
