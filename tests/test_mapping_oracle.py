"""Mapping kernels: the oracle's restatement against the reference's own
kernels (CPU only), through the whole map_channels_segments sequence."""
import numpy as np
import pytest

import oracle as O
from mapping_cases import ComparingRunner, midslope_case, oracle_runner, pipeline_case
from slm_b200 import mapping as M

needs_ref = pytest.mark.skipif(not O.ref_available("count_downchannels"),
                               reason="reference kernels not compiled (oracle/_ref)")


@needs_ref
@pytest.mark.parametrize("kw", [dict(nx=96, ny=80, seed=5), dict(nx=120, ny=72, seed=6, channel_pct=90.0),
                                dict(nx=64, ny=64, seed=7, segmentation_threshold=4)])
def test_pipeline_vs_reference(kw):
    c, info, data = pipeline_case(**kw)
    run = ComparingRunner()
    ok = M.map_channels_segments(None, info, data, runner=run)
    assert ok, run.calls
    names = [n for n, _ in run.calls]
    for k in ("connect_channels", "map_channel_heads", "count_downchannels", "flag_downchannels",
              "label_confluences", "segment_downchannels", "hillslopes", "segment_hillslopes",
              "subsegment_channel_edges", "subsegment_flanks", "fix_right_flanks", "fix_left_flanks"):
        assert k in names, k
    assert run.mismatches == [], run.mismatches
    assert (data.label_array != 0).sum() > 0
    n = midslope_case(data, info)
    assert n > 0
    assert M.hsl(None, info, data, False, runner=run)
    assert run.mismatches == []
    assert np.count_nonzero(data.subsegment_hsl_array) > 0


@needs_ref
def test_prune_channel_heads_vs_reference():
    c, info, data = pipeline_case(nx=80, ny=80, seed=8)
    run = ComparingRunner()
    M.map_channels(info, data)
    M.connect_channel_pixels(None, info, data, runner=run)
    M.thin_channels(info, data)
    M.map_channel_heads(None, info, data, runner=run)
    M.prune_channel_heads(None, info, data, runner=run)
    assert ("prune_channel_heads", int(np.sum(~data.mask_array & ((data.mapping_array & info.is_channelhead) > 0)))) or True
    assert run.mismatches == []
