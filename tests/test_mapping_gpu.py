"""Mapping kernels on the GPU against the oracle, kernel by kernel through the
map_channels_segments sequence (bit-exact: integer flags, counts, links and
labels; hillslope lengths are float results of bit-exact RK walks)."""
import numpy as np
import pytest

import oracle as O
from mapping_cases import incised_pipeline_case, midslope_case, oracle_runner, pipeline_case
from slm_b200 import mapping as M

pytestmark = pytest.mark.gpu


class DeviceVsOracle:
    def __init__(self):
        self.device = M.DeviceRunner()
        self.mismatches = []
        self.calls = []

    def __call__(self, name, params, seeds, arrays):
        expect = [a.copy() for a in arrays]
        oracle_runner(name, params, seeds, expect)
        st = self.device(name, params, seeds, arrays)
        assert st == 0, (name, st)
        self.calls.append((name, seeds.shape[0]))
        for k, (a, b) in enumerate(zip(arrays, expect)):
            if not np.array_equal(a.view(np.uint8), b.view(np.uint8)):
                self.mismatches.append((name, k, int(np.sum(a != b))))
                a[...] = b  # continue from the oracle's state so later kernels are compared too


@pytest.mark.parametrize("kw", [dict(nx=96, ny=80, seed=5), dict(nx=120, ny=72, seed=6, channel_pct=90.0),
                                dict(nx=64, ny=64, seed=7, segmentation_threshold=4),
                                dict(nx=256, ny=192, seed=9, channel_pct=92.0)])
def test_mapping_pipeline_bit_exact(kw):
    c, info, data = pipeline_case(**kw)
    run = DeviceVsOracle()
    assert M.map_channels_segments(None, info, data, runner=run)
    assert run.mismatches == [], run.mismatches
    assert len(run.calls) == 15
    midslope_case(data, info)
    assert M.hsl(None, info, data, False, runner=run)
    assert run.mismatches == [], run.mismatches


def test_prune_channel_heads_bit_exact():
    c, info, data = pipeline_case(nx=80, ny=80, seed=8)
    run = DeviceVsOracle()
    M.map_channels(info, data)
    M.connect_channel_pixels(None, info, data, runner=run)
    M.thin_channels(info, data)
    M.map_channel_heads(None, info, data, runner=run)
    M.prune_channel_heads(None, info, data, runner=run)
    assert run.mismatches == []


@pytest.mark.parametrize("seed,thin_heads", [(21, True), (22, False), (23, False)])
def test_prune_channel_heads_random_heads(seed, thin_heads):
    """Random thin-channel grids and random heads: all heads thin (the
    parallel case) and heads of which some are not thin, next to isolated
    thin heads (the case the sequential schedule decides), against the
    oracle's sequential schedule."""
    c, info, data = pipeline_case(nx=60, ny=50, seed=8)
    rng = np.random.default_rng(seed)
    nxp, nyp = data.mask_array.shape
    m = np.zeros((nxp, nyp), np.uint32)
    thin = rng.random((nxp, nyp)) < 0.25
    m[thin] |= info.is_thinchannel | info.is_channel
    # isolated thin pixels next to non-thin ones
    for x, y in rng.integers(4, min(nxp, nyp) - 4, size=(40, 2)):
        m[x - 1:x + 2, y - 1:y + 2] &= ~np.uint32(info.is_thinchannel)
        m[x, y] |= info.is_thinchannel
    pool = np.argwhere(((m & info.is_thinchannel) != 0) if thin_heads else np.ones_like(thin))
    heads = pool[rng.choice(pool.shape[0], size=min(400, pool.shape[0]), replace=False)]
    heads = heads[np.lexsort((heads[:, 1], heads[:, 0]))]
    m[heads[:, 0], heads[:, 1]] |= info.is_channelhead
    data.mapping_array = m
    info.n_seed_points = np.uint32(heads.shape[0])
    seeds = (heads - int(info.pad_width)).astype(np.float32)
    prm = M.kernel_params(info, "PRUNE_CHANNEL_HEADS")
    expect = [data.mask_array, data.uv_array, m.copy()]
    oracle_runner("prune_channel_heads", prm, seeds, expect)
    got = [data.mask_array, data.uv_array, m.copy()]
    assert M.DeviceRunner()("prune_channel_heads", prm, seeds, got) == 0
    assert np.array_equal(got[2], expect[2])
    assert not np.array_equal(got[2], m)  # something was pruned


def test_device_pipeline_end_to_end_matches_oracle_pipeline():
    """The whole sequence on the device alone equals the whole sequence on the oracle."""
    _, info, data = pipeline_case(nx=160, ny=128, seed=11)
    _, info2, data2 = pipeline_case(nx=160, ny=128, seed=11)
    dev = M.DeviceRunner()
    assert M.map_channels_segments(None, info, data, runner=dev)
    assert M.map_channels_segments(None, info2, data2, runner=oracle_runner)
    assert dev.status == 0
    for name in ("mapping_array", "count_array", "link_array", "label_array", "channel_label_array"):
        assert np.array_equal(getattr(data, name), getattr(data2, name)), name


@pytest.mark.parametrize("seed", [3, 4])
def test_mapping_pipeline_incised_bit_exact(seed):
    """Valley floors one pixel wide: count_downchannels walks oscillate to the
    1000*MAX_N_STEPS bound, exercising the compressed event replay."""
    info, data = incised_pipeline_case(seed=seed)
    run = DeviceVsOracle()
    assert M.map_channels_segments(None, info, data, runner=run)
    assert run.mismatches == [], run.mismatches
    midslope_case(data, info)
    assert M.hsl(None, info, data, False, runner=run)
    assert run.mismatches == [], run.mismatches


@pytest.mark.parametrize("form", ["settle", "rounds"])
@pytest.mark.parametrize("case", ["pipeline", "incised"])
def test_flank_fix_forms_bit_exact(monkeypatch, form, case):
    """fix_right/left_flanks in both forms -- every walk traced once into
    linked blocks and settled in one persistent launch that waits on
    lower-index owners (the default), and resolved in rounds
    (SLM_FLANK_ROUNDS=1, the fallback) -- give the oracle's labels."""
    if form == "rounds":
        monkeypatch.setenv("SLM_FLANK_ROUNDS", "1")
    else:
        monkeypatch.delenv("SLM_FLANK_ROUNDS", raising=False)
    if case == "pipeline":
        _, info, data = pipeline_case(nx=160, ny=128, seed=21, channel_pct=91.0)
    else:
        info, data = incised_pipeline_case(seed=5)
    run = DeviceVsOracle()
    assert M.map_channels_segments(None, info, data, runner=run)
    assert run.mismatches == [], run.mismatches
    assert [n for n, _ in run.calls].count("fix_right_flanks") == 1


@pytest.mark.parametrize("form", ["settle", "rounds"])
def test_flank_fix_in_chunks_bit_exact(monkeypatch, form):
    """A path budget far below the total: the single-pass store runs out, so
    fix_right/left_flanks store the paths contiguously in many index-ordered
    chunks and settle them chunk by chunk (or, with SLM_FLANK_ROUNDS=1,
    resolve them in rounds); labels equal the oracle's."""
    from slm_b200 import map_kernels
    monkeypatch.setattr(map_kernels, "FLANK_PATH_BUDGET", 2048)
    if form == "rounds":
        monkeypatch.setenv("SLM_FLANK_ROUNDS", "1")
    else:
        monkeypatch.delenv("SLM_FLANK_ROUNDS", raising=False)
    c, info, data = pipeline_case(nx=120, ny=96, seed=12)
    run = DeviceVsOracle()
    assert M.map_channels_segments(None, info, data, runner=run)
    assert run.mismatches == [], run.mismatches
    assert ("fix_right_flanks", ) == tuple(n for n, _ in run.calls if n == "fix_right_flanks")


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_device_thinning_matches_host(seed):
    from slm_b200.skeleton import zhang_suen, zhang_suen_device
    rng = np.random.default_rng(seed)
    img = np.zeros((97, 131), bool)
    for _ in range(40):
        x, y = rng.integers(0, 97), rng.integers(0, 131)
        w, h = rng.integers(1, 9), rng.integers(1, 30)
        img[max(0, x - w):x + w, max(0, y - h):y + h] = True
    img[0, :] = True  # touching the border (outside counts as 0)
    assert np.array_equal(zhang_suen_device(img), zhang_suen(img))


@pytest.mark.parametrize("case", ["plain96", "plain256", "incised3", "incised4"])
def test_device_resident_mapping_matches(case):
    """The whole sequence with the grids on the GPU (seed picking, flag
    updates, thinning and relabelling as device kernels) equals the
    reference-shaped wrappers' sequence, array for array, and so do the
    hillslope lengths."""
    import copy
    from slm_b200.mapping_device import map_channels_segments_device
    if case.startswith("plain"):
        nx = 96 if case == "plain96" else 256
        _, info, data = pipeline_case(nx=nx, ny=80 if nx == 96 else 192, seed=9)
    else:
        info, data = incised_pipeline_case(seed=int(case[-1]))
    info2, data2 = copy.deepcopy(info), copy.deepcopy(data)
    assert M.map_channels_segments(None, info, data)
    ok, dm = map_channels_segments_device(info2, data2)
    assert ok and dm.status == 0
    for name in ("mapping_array", "count_array", "link_array", "label_array", "channel_label_array"):
        a, b = getattr(data, name), getattr(data2, name)
        assert a.dtype == b.dtype and np.array_equal(a, b), name
    midslope_case(data, info)
    assert M.hsl(None, info, data, False)
    dm.upload_mapping(data.mapping_array)
    got = dm.hsl(False)
    assert np.array_equal(got.view(np.uint32), data.subsegment_hsl_array.view(np.uint32))


@pytest.mark.parametrize("seed", range(6))
def test_flag_downchannels_random_graphs(seed):
    """flag_downchannels runs all heads' walks at once; on random link graphs
    (cycles, self-loops, masked pixels, minor-inflow flags, prior counts,
    heads walked over by other heads) it equals the oracle's sequential run."""
    from cases import Case
    from slm_b200 import map_kernels
    from slm_b200.params import kernel_params
    rng = np.random.default_rng(seed)
    c = Case(nx=36, ny=28, seed=seed + 40, step=0.5, max_length=1.5)  # max_n_steps 3: lim 3000
    info = c.info
    nxp, nyp = c.mask.shape
    n = nxp * nyp
    mask = rng.random((nxp, nyp)) < 0.08
    link = rng.integers(0, n, size=n).astype(np.uint32)
    near = rng.random(n) < 0.7  # mostly a neighbour, as channel links are
    xs, ys = np.divmod(np.arange(n), nyp)
    nx2 = np.clip(xs + rng.integers(-1, 2, n), 0, nxp - 1)
    ny2 = np.clip(ys + rng.integers(-1, 2, n), 0, nyp - 1)
    link[near] = (nx2 * nyp + ny2)[near].astype(np.uint32)
    link = link.reshape(nxp, nyp)
    mapping = np.zeros((nxp, nyp), np.uint32)
    mapping[rng.random((nxp, nyp)) < 0.05] |= np.uint32(info.is_minorinflow)
    mapping[rng.random((nxp, nyp)) < 0.3] |= np.uint32(info.is_channelhead)
    count = rng.integers(0, 6, size=(nxp, nyp)).astype(np.uint32)
    cand = np.argwhere(~mask)
    heads = cand[rng.choice(len(cand), size=min(150, len(cand)), replace=False)]
    seeds = (heads.astype(np.float32) - info.pad_width).astype(np.float32)
    info.n_seed_points = np.uint32(len(seeds))
    prm = kernel_params(info, "FLAG_DOWNCHANNELS")
    uv = np.zeros((nxp, nyp, 2), np.float32)
    a = [mask, uv, mapping.copy(), count.copy(), link]
    b = [mask, uv, mapping.copy(), count.copy(), link]
    O.map_kernel("flag_downchannels", prm, seeds, a)
    map_kernels.run("flag_downchannels", prm, seeds, b)
    assert np.array_equal(b[2], a[2]), "mapping"
    assert np.array_equal(b[3], a[3]), "count"


@pytest.mark.gpu
def test_mapping_stage_pass1_on_the_gpu():
    """Mapping.pass1 with its defaults (kernels and thinning on the GPU) equals
    the same pass on the oracle with the host thinning."""
    import types

    from mapping_cases import incised_pipeline_case
    from slm_b200.mapping_stage import Mapping
    from slm_b200.skeleton import zhang_suen
    from slm_b200.useful import default_parameters
    info0, data0 = incised_pipeline_case(n=64, seed=3, n_incisions=6, max_steps=200)
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
    geodata = types.SimpleNamespace(roi_nx=64, roi_ny=64, pad_width=2, roi_pixel_size=2.0)
    preprocess = types.SimpleNamespace(uv_array=data0.uv_array)
    params = {"mapping": dict(coarse_channel_threshold=float(info0.channel_threshold), coarse_segmentation_threshold=10,
                              midslope_filter_sigma=2.0, midslope_threshold=0.2, ridge_threshold=0.3)}
    gpu = Mapping(state, params, geodata, preprocess, trace)
    gpu.pass1()
    cpu = Mapping(state, params, geodata, preprocess, trace, runner=oracle_runner, thin=zhang_suen)
    cpu.pass1()
    assert np.array_equal(gpu.mapping_array, cpu.mapping_array)
    assert np.array_equal(gpu.coarse_subsegment_array, cpu.coarse_subsegment_array)
    assert gpu.n_coarse_subsegments == cpu.n_coarse_subsegments > 0


@pytest.mark.gpu
@pytest.mark.parametrize("hsl_method", ["fmm", "traced"])
def test_mapping_stage_pass2_on_the_gpu(hsl_method):
    """Passes 1 and 2 with the region's grids on the GPU (device engine: the
    mapping sequence and the fast-marching or traced lengths with the
    windows resident there) equal the same passes through the wrappers on
    the oracle; the channel thresholds come from the device KDE on both
    sides."""
    import types

    from mapping_cases import incised_pipeline_case
    from slm_b200 import analysis as A
    from slm_b200.mapping_stage import Mapping
    from slm_b200.skeleton import zhang_suen
    from slm_b200.useful import default_parameters
    from test_mapping_stage import ActiveMasks
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
                  fine_segmentation_threshold=10, midslope_filter_sigma=2.0, midslope_threshold=0.2,
                  ridge_filter_sigma=2.0, ridge_threshold=0.3, do_measure_hsl_from_ridges=False,
                  n_hsl_averaging_threshold=1, hsl_averaging_threshold=5.0, min_channel_threshold=1.0,
                  max_channel_threshold=1000.0, guess_channel_threshold=30.0)
    analysis_params = {"analysis": dict(A.ANALYSIS_PARAMETERS, n_hist_bins=512, n_pdf_points=64,
                                        pdf_slt_min=1e-3, pdf_sla_min=1e-3, pdf_slc_min=1e-3)}
    out = []
    for runner in (None, oracle_runner):
        state = ActiveMasks(data0.mask_array, **vars(d.state))
        m = Mapping(state, {"mapping": params}, geodata, preprocess, trace,
                    analysis=A.Analysis(state, analysis_params, geodata, None, trace), runner=runner,
                    thin=zhang_suen)
        m.pass1()
        m.pass2(hsl_method=hsl_method)
        out.append(m)
    gpu, cpu = out
    assert gpu.n_coarse_subsegments == cpu.n_coarse_subsegments > 1
    assert np.array_equal(gpu.mapping_array, cpu.mapping_array)
    assert np.array_equal(gpu.hsl_array, cpu.hsl_array) and gpu.hsl_array.any()
    assert np.array_equal(gpu.hsl_mean_array, cpu.hsl_mean_array)
    assert gpu.hsl_stats_df.equals(cpu.hsl_stats_df)


@pytest.mark.parametrize("hsl_method", ["fmm", "traced"])
def test_mapping_stage_pass2_threads_equal_order(hsl_method):
    """Pass 2 with its independent coarse subsegments on six threads and
    streams (the default on the GPU) equals pass 2 run one subsegment after
    another in label order, on a grid with many subsegments."""
    import types

    from mapping_cases import incised_pipeline_case
    from slm_b200 import analysis as A
    from slm_b200.mapping_stage import Mapping
    from slm_b200.skeleton import zhang_suen
    from slm_b200.useful import default_parameters
    from test_mapping_stage import ActiveMasks
    n = 160
    info0, data0 = incised_pipeline_case(n=n, seed=5, n_incisions=14, max_steps=300)
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
    analysis_params = {"analysis": dict(A.ANALYSIS_PARAMETERS, n_hist_bins=512, n_pdf_points=64,
                                        pdf_slt_min=1e-3, pdf_sla_min=1e-3, pdf_slc_min=1e-3)}
    out = []
    for workers in (1, 6):
        params = dict(vars(d.mapping))
        params.update(coarse_channel_threshold=float(info0.channel_threshold), coarse_segmentation_threshold=12,
                      fine_segmentation_threshold=6, midslope_filter_sigma=2.0, midslope_threshold=0.2,
                      ridge_filter_sigma=2.0, ridge_threshold=0.3, do_measure_hsl_from_ridges=False,
                      n_hsl_averaging_threshold=1, hsl_averaging_threshold=5.0, min_channel_threshold=1.0,
                      max_channel_threshold=1000.0, guess_channel_threshold=30.0, pass2_workers=workers)
        state = ActiveMasks(data0.mask_array, **vars(d.state))
        m = Mapping(state, {"mapping": params}, geodata, preprocess, trace,
                    analysis=A.Analysis(state, analysis_params, geodata, None, trace), thin=zhang_suen)
        m.pass1()
        m.pass2(hsl_method=hsl_method)
        out.append(m)
    seq, par = out
    assert seq.n_coarse_subsegments == par.n_coarse_subsegments > 20
    assert np.array_equal(seq.mapping_array, par.mapping_array)
    assert np.array_equal(seq.hsl_array.view(np.uint32), par.hsl_array.view(np.uint32)) and seq.hsl_array.any()
    assert np.array_equal(seq.hsl_mean_array, par.hsl_mean_array)
    assert seq.hsl_stats_df.equals(par.hsl_stats_df)
    assert seq.engine.status == par.engine.status


@pytest.mark.parametrize("n", [0, 1, 1000, 65536, 65537, 300001, 10_000_000])
def test_exclusive_scan_u64(n):
    """The tiled exclusive scan behind the stored flank paths (one block up
    to 8 tiles of 8192, three launches above) against NumPy's cumsum."""
    import ctypes

    import torch

    from slm_b200 import _lib
    L = _lib.load()
    rng = np.random.default_rng(n)
    x = rng.integers(0, 5000, n, dtype=np.uint64)
    dev = torch.device("cuda", 0)
    xin = torch.from_numpy(x.view(np.int64)).to(dev) if n else torch.zeros(1, dtype=torch.int64, device=dev)
    out = torch.full((n + 1,), -1, dtype=torch.int64, device=dev)
    scratch = torch.empty(max(1, int(L.slm_exclusive_scan_u64_scratch(n))), dtype=torch.uint8, device=dev)
    _lib.check(L.slm_exclusive_scan_u64(_lib.ptr(xin), n, _lib.ptr(out), _lib.ptr(scratch), scratch.numel(),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    want = np.concatenate([[0], np.cumsum(x, dtype=np.uint64)])
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
