"""Mapping.pass1 against the reference's own Mapping.pass1 (CPU only).

Both sides run every mapping kernel through the oracle (the reference's
wrapper modules are stood in by this package's wrappers with the oracle
runner), and both thin with this package's host thinning (scikit-image is
absent).  So what is compared is pass 1 itself: the crop, the midslope and
ridge flags, the reference's map_channels_segments sequence, the coarse
subsegments and their mask, and the flag merge."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

from mapping_cases import incised_pipeline_case, oracle_runner
from slm_b200 import mapping as M
from slm_b200.mapping_stage import Mapping
from slm_b200.skeleton import zhang_suen
from slm_b200.useful import default_parameters
from test_params import _load_reference_modules


def _reference_mapping_module(reference_dir):
    mods = _load_reference_modules(reference_dir)
    names = ["skimage", "skimage.morphology", "skimage.filters", "skimage.filters.rank", "skfmm", "streamlines",
             "streamlines.core", "streamlines.useful", "streamlines.pocl"] + \
        ["streamlines." + n for n in ("connect", "channelheads", "countlink", "label", "segment", "hillslopes",
                                      "lengths")]
    saved = {k: sys.modules.get(k) for k in names}
    st = {k: types.ModuleType(k) for k in names}
    st["skimage.morphology"].skeletonize = zhang_suen
    st["skimage.morphology"].medial_axis = lambda a: a  # both sides thin once, with the same thinning
    st["skimage.morphology"].thin = st["skimage.morphology"].disk = None
    st["skimage.filters"].gaussian = None
    st["skimage.filters.rank"].mean = st["skimage.filters.rank"].median = None
    st["streamlines.core"].Core = type("Core", (), {})
    st["streamlines.pocl"].Initialize_cl = None

    def bind(fn):
        return lambda cl_state, info, data, verbose=False, **kw: fn(cl_state, info, data, verbose, runner=oracle_runner,
                                                                   **kw)
    st["streamlines.connect"].connect_channel_pixels = bind(M.connect_channel_pixels)
    st["streamlines.channelheads"].map_channel_heads = bind(M.map_channel_heads)
    st["streamlines.channelheads"].prune_channel_heads = bind(M.prune_channel_heads)
    st["streamlines.countlink"].count_downchannels = bind(M.count_downchannels)
    st["streamlines.countlink"].flag_downchannels = bind(M.flag_downchannels)
    st["streamlines.label"].label_confluences = bind(M.label_confluences)
    st["streamlines.segment"].segment_channels = bind(M.segment_channels)
    st["streamlines.segment"].segment_hillslopes = bind(M.segment_hillslopes)
    st["streamlines.segment"].subsegment_flanks = bind(M.subsegment_flanks)
    st["streamlines.hillslopes"].link_hillslopes = bind(M.link_hillslopes)
    for n in ("connect", "channelheads", "countlink", "label", "segment", "hillslopes", "lengths"):
        setattr(st["streamlines"], n, st["streamlines." + n])
    sys.modules.update(st)
    sys.modules["streamlines.useful"] = mods["useful"]
    if not hasattr(np, "bool"):
        np.bool = np.bool_
    try:
        spec = importlib.util.spec_from_file_location(
            "reference_mapping_stage", os.path.join(reference_dir, "python", "streamlines", "mapping.py"))
        mod = importlib.util.module_from_spec(spec)
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


@pytest.mark.parametrize("seed,do_map_hsl", [(3, True), (5, False)])
def test_pass1_matches_reference(reference_dir, seed, do_map_hsl):
    R = _reference_mapping_module(reference_dir)
    n = 64
    info0, data0 = incised_pipeline_case(n=n, seed=seed, n_incisions=6, max_steps=200)
    slt, slc = data0.slt_array, data0.slc_array
    with np.errstate(divide="ignore", invalid="ignore"):
        sla = np.where(slc > 0, np.sqrt(2.0) * slt / slc, 0.0).astype(np.float32)
    d = default_parameters()
    trace = types.SimpleNamespace(**vars(d.trace))
    trace.subpixel_seed_point_density, trace.jitter_magnitude = 1, 0.0
    trace.integrator_step_factor, trace.max_length = 0.1, 20.0
    trace.slc_array, trace.slt_array, trace.sla_array = slc, slt, sla
    mask = data0.mask_array.copy()
    state = types.SimpleNamespace(**vars(d.state))
    state.reset_active_masks = lambda: None
    state.merge_active_masks = lambda: mask.copy()
    geodata = types.SimpleNamespace(roi_nx=n, roi_ny=n, pad_width=2, roi_pixel_size=2.0)
    preprocess = types.SimpleNamespace(uv_array=data0.uv_array)
    params = dict(vars(d.mapping))
    params.update(coarse_channel_threshold=float(info0.channel_threshold), coarse_segmentation_threshold=10,
                  fine_segmentation_threshold=10, do_map_channels_segments=True, do_map_hsl=do_map_hsl,
                  midslope_filter_sigma=2.0, midslope_threshold=0.2, ridge_filter_sigma=2.0, ridge_threshold=0.3,
                  do_measure_hsl_from_ridges=False)
    class Info(R.Info):  # NumPy 1.x widened int32 + 2**31 to int64; NumPy 2 raises instead
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.left_flank_addition = np.int64(self.left_flank_addition)
    R.Info = Info
    ref = R.Mapping.__new__(R.Mapping)
    ref.__dict__.update(params)
    ref.__dict__.update(state=state, geodata=geodata, preprocess=preprocess, trace=trace, cl_state=None,
                        verbose=False, vprogress=False, vbackup=False, print=lambda *a, **k: None)
    ref.pass1()
    mine = Mapping(state, {"mapping": params}, geodata, preprocess, trace, runner=oracle_runner, thin=zhang_suen)
    mine.pass1()
    assert np.array_equal(mine.mapping_array, ref.mapping_array)
    assert np.array_equal(mine.coarse_subsegment_array, ref.coarse_subsegment_array)
    assert np.array_equal(mine.coarse_subsegments_list_array, ref.coarse_subsegments_list_array)
    assert np.array_equal(mine.merged_coarse_mask_array, ref.merged_coarse_mask_array)
    info = mine.info
    assert mine.n_coarse_subsegments > 0
    assert ((mine.mapping_array & info.is_midslope) > 0).any() and ((mine.mapping_array & info.is_ridge) > 0).any()


@pytest.mark.parametrize("seed", [3, 4])
def test_traced_hillslope_length_statistics_match_reference(reference_dir, seed):
    """The traced lengths of the midslope pixels (the lengths kernel on the
    oracle), their per-subsegment statistics (length_statistics) and the
    painted means (paint_means) against the reference's select_subsegments,
    measure_hsl_traced, parse_hsl and remap_hsl on the same mapped grids."""
    import copy

    import torch

    from mapping_cases import midslope_case
    from slm_b200 import mapping_stage as MS
    R = _reference_mapping_module(reference_dir)
    R.lengths.hsl = lambda cl_state, info, data, do_use_ridges, verbose=False: M.hsl(
        cl_state, info, data, do_use_ridges, verbose, runner=oracle_runner)
    info, data = incised_pipeline_case(n=64, seed=seed, n_incisions=6, max_steps=200)
    assert M.map_channels_segments(None, info, data, runner=oracle_runner)
    midslope_case(data, info, seed=seed, frac=0.08)
    info.coarse_label = 7
    params = dict(do_measure_hsl_from_ridges=False, n_hsl_averaging_threshold=2, hsl_averaging_threshold=5.0)
    ref = R.Mapping.__new__(R.Mapping)
    ref.__dict__.update(params, cl_state=None, verbose=False, print=lambda *a, **k: None)
    rd = copy.deepcopy(data)
    ref.select_subsegments(info, rd)
    assert ref.measure_hsl_traced(info, rd)
    assert ref.parse_hsl(info, rd)
    assert ref.remap_hsl(info, rd)
    # the same through this package: the engine's lengths, then the statistics
    md = copy.deepcopy(data)
    picked = ((md.mapping_array & info.is_midslope) > 0) & ~md.mask_array
    fine = md.label_array[picked]
    engine = MS.WrapperEngine(oracle_runner)
    engine.data = md
    lengths = engine.lengths(info, torch.from_numpy(md.mapping_array.astype(np.int64)), int(fine.shape[0]))
    assert np.array_equal(lengths.view(np.uint32), rd.subsegment_hsl_array.view(np.uint32))
    stats = MS.length_statistics(fine, lengths, 7)
    assert stats.equals(rd.hsl_stats_df)
    painted = MS.paint_means(torch.from_numpy(md.label_array), stats, 2, "cpu").numpy()
    assert np.array_equal(painted, rd.hsl_array)
    kept = painted[~np.isnan(painted)]
    assert np.mean(kept[kept >= 5.0]) == rd.trace_mean_hsl
    assert len(stats) > 3 and painted.any()


@pytest.mark.parametrize("seed", [3, 5])
def test_fmm_lengths_match_reference(reference_dir, seed, monkeypatch):
    """The wrappers' fmm_lengths (the oracle's solver) against the reference's
    own select_subsegments(do_restrict=False) + Mapping.fmm_lengths, with
    skfmm.distance stood in by the oracle's restatement, on the same mapped
    grids: the int32 lengths per selected subsegment and their mean."""
    import copy

    import eikonal
    R = _reference_mapping_module(reference_dir)
    monkeypatch.setattr(R, "skfmm", types.SimpleNamespace(distance=eikonal.distance), raising=False)
    info, data = incised_pipeline_case(n=64, seed=seed, n_incisions=6, max_steps=200)
    assert M.map_channels_segments(None, info, data, runner=oracle_runner)
    ref = R.Mapping.__new__(R.Mapping)
    ref.__dict__.update(do_measure_hsl_from_ridges=False, cl_state=None, verbose=False, print=lambda *a, **k: None,
                        geodata=types.SimpleNamespace(roi_pixel_size=2.0))
    rd = copy.deepcopy(data)
    ref.select_subsegments(info, rd, do_restrict=False)
    ok = ref.fmm_lengths(info, rd)
    md = copy.deepcopy(data)
    md.selected_subsegments_array = rd.selected_subsegments_array.copy()
    assert M.fmm_lengths(None, info, md, 2.0, runner=oracle_runner) == ok
    assert md.subsegment_hsl_array.dtype == rd.subsegment_hsl_array.dtype == np.int32
    assert np.array_equal(md.subsegment_hsl_array, rd.subsegment_hsl_array)
    assert ok and md.fmm_mean_hsl == rd.fmm_mean_hsl
    assert (md.subsegment_hsl_array > 0).sum() > 3


class ActiveMasks:
    """The reference State's active-mask bookkeeping (state.py:374-459)."""

    def __init__(self, dtm_mask, **params):
        self.__dict__.update(params)
        self.verbose = False
        self.active_masks_dict = {"dtm": dtm_mask.copy()}

    def add_active_mask(self, item):
        if list(item.keys())[0] not in self.active_masks_dict:
            self.active_masks_dict.update(item)

    def remove_active_mask(self, name):
        self.active_masks_dict.pop(name, None)

    def reset_active_masks(self):
        self.active_masks_dict = {k: v for k, v in self.active_masks_dict.items() if k in ("dtm", "basin", "uv")}

    def merge_active_masks(self, out=None):
        for k, m in enumerate(self.active_masks_dict.values()):
            if k == 0:
                if out is None:
                    out = m.copy()
                else:
                    np.copyto(out, m)
            else:
                out |= m
        return out


def _pass2_against_reference(reference_dir, monkeypatch, hsl_method):
    """Runs the reference's pass1 + pass2 and this package's on the same
    incised case (kernels on the oracle; channel thresholds from the same
    Analysis on a CPU stand-in KDE); returns (reference, mine)."""
    import pandas as pd

    from slm_b200 import analysis as A
    from test_analysis_stage import fake_bivariate, fake_univariate
    monkeypatch.setattr(A.kde, "estimate_univariate_pdf", fake_univariate)
    monkeypatch.setattr(A.kde, "estimate_bivariate_pdf", fake_bivariate)
    if not hasattr(pd.DataFrame, "append"):  # the reference's DataFrame.append (pandas < 2)
        monkeypatch.setattr(pd.DataFrame, "append", lambda self, other: pd.concat([self, other]), raising=False)
    R = _reference_mapping_module(reference_dir)
    R.lengths.hsl = lambda cl_state, info, data, do_use_ridges, verbose=False: M.hsl(
        cl_state, info, data, do_use_ridges, verbose, runner=oracle_runner)

    class Info(R.Info):  # NumPy 1.x widened int32 + 2**31 to int64; NumPy 2 raises instead
        def __init__(self, *a, **k):
            super().__init__(*a, **k)
            self.left_flank_addition = np.int64(self.left_flank_addition)
    R.Info = Info
    n = 64
    info0, data0 = incised_pipeline_case(n=n, seed=3, n_incisions=6, max_steps=200)
    slt, slc = data0.slt_array, data0.slc_array
    with np.errstate(divide="ignore", invalid="ignore"):
        sla = np.where(slc > 0, np.sqrt(2.0) * slt / slc, 0.0).astype(np.float32)
    d = default_parameters()
    trace = types.SimpleNamespace(**vars(d.trace))
    trace.subpixel_seed_point_density, trace.jitter_magnitude = 1, 0.0
    trace.integrator_step_factor, trace.max_length = 0.1, 20.0
    trace.slc_array, trace.slt_array, trace.sla_array = slc, slt, sla
    geodata = types.SimpleNamespace(roi_nx=n, roi_ny=n, pad_width=2, roi_pixel_size=2.0)
    preprocess = types.SimpleNamespace(uv_array=data0.uv_array)
    params = dict(vars(d.mapping))
    params.update(coarse_channel_threshold=float(info0.channel_threshold), coarse_segmentation_threshold=40,
                  fine_segmentation_threshold=10, do_map_channels_segments=True, do_map_hsl=True,
                  midslope_filter_sigma=2.0, midslope_threshold=0.2, ridge_filter_sigma=2.0, ridge_threshold=0.3,
                  do_measure_hsl_from_ridges=False, n_hsl_averaging_threshold=1, hsl_averaging_threshold=5.0,
                  min_channel_threshold=1.0, max_channel_threshold=1000.0, guess_channel_threshold=30.0)
    # log limits low enough that every subsegment has data (with none, the
    # reference's distribution raises and its pass 2 stops)
    analysis_params = {"analysis": dict(A.ANALYSIS_PARAMETERS, n_hist_bins=512, n_pdf_points=64,
                                        pdf_slt_min=1e-3, pdf_sla_min=1e-3, pdf_slc_min=1e-3)}

    ref_state = ActiveMasks(data0.mask_array, **vars(d.state))
    ref = R.Mapping.__new__(R.Mapping)
    ref.__dict__.update(params)
    ref.__dict__.update(state=ref_state, geodata=geodata, preprocess=preprocess, trace=trace, cl_state=None,
                        verbose=False, vprogress=False, vbackup=False, print=lambda *a, **k: None,
                        analysis=A.Analysis(ref_state, analysis_params, geodata, None, trace))
    if hsl_method == "traced":
        ref.select_subsegments = lambda info, data, do_restrict=True: R.Mapping.select_subsegments(ref, info, data)

        def traced(info, data):
            data.fmm_mean_hsl = 0.0
            return R.Mapping.measure_hsl_traced(ref, info, data)
        ref.measure_hsl_fmm = traced
        ref.remap_hsl = lambda info, data, n_hsl_averaging_threshold=None: R.Mapping.remap_hsl(ref, info, data)
    else:  # the reference's own fast-marching branch, skfmm's distance from the oracle
        import eikonal
        monkeypatch.setattr(R, "skfmm", types.SimpleNamespace(distance=eikonal.distance), raising=False)
    ref.pass1()
    ref.pass2()

    my_state = ActiveMasks(data0.mask_array, **vars(d.state))
    mine = Mapping(my_state, {"mapping": params}, geodata, preprocess, trace,
                   analysis=A.Analysis(my_state, analysis_params, geodata, None, trace), runner=oracle_runner,
                   thin=zhang_suen)
    mine.pass1()
    mine.pass2(hsl_method=hsl_method)
    return ref, mine


def _assert_same_pass2(ref, mine):
    assert mine.n_coarse_subsegments == ref.n_coarse_subsegments > 1
    assert np.array_equal(mine.mapping_array, ref.mapping_array)
    assert np.array_equal(mine.hsl_array, ref.hsl_array) and mine.hsl_array.any()
    assert np.array_equal(mine.hsl_mean_array, ref.hsl_mean_array) and mine.hsl_mean_array.size > 0
    assert mine.hsl_stats_df.equals(ref.hsl_stats_df)


def test_pass2_traced_matches_reference(reference_dir, monkeypatch):
    """Pass 2 with the lengths traced along streamlines, against the
    reference's pass2 with its fast-marching measurement swapped for its own
    traced-length methods (the alternative it keeps switched off)."""
    _assert_same_pass2(*_pass2_against_reference(reference_dir, monkeypatch, "traced"))


def test_pass2_fmm_matches_reference(reference_dir, monkeypatch):
    """Pass 2 as the reference runs it: its own fast-marching branch
    (select_subsegments without restriction, fmm_lengths, parse_hsl,
    remap_hsl with no count threshold), skfmm.distance stood in by the
    oracle's restatement, against this package's default pass 2 with the
    oracle's solver.  Pins the call site: the grown regions, the channel
    phi, the ratio test, the doubled mean and its int32 truncation, the
    painting and the statistics."""
    ref, mine = _pass2_against_reference(reference_dir, monkeypatch, "fmm")
    _assert_same_pass2(ref, mine)
    assert (mine.hsl_array > 0).sum() > 100

