"""The drop-in stage wrappers (Trajectories, Fields) on the GPU against the oracle."""
import numpy as np
import pytest

import oracle as O
from cases import Case
from slm_b200.fields import Fields
from slm_b200.trajectories import Trajectories
from slm_b200.useful import Data, compute_stats, create_seeds

pytestmark = pytest.mark.gpu


def _data(c, stats=None):
    return Data(info=c.info, mask_array=c.mask, uv_array=c.uv,
                mapping_array=np.zeros(c.mask.shape, np.uint32), traj_stats_df=stats)


@pytest.mark.parametrize("integrator", [2, 4])
def test_trajectories_stage(integrator):
    c = Case(nx=64, ny=48, seed=81, step=0.25, max_length=80.0, n_traj_seeds=300)
    tr = Trajectories(0, 0, info=c.info, data=_data(c), integrator=integrator)
    tr.integrate()
    n = int(c.info.n_seed_points)
    for d, sign in ((0, np.float32(1.0)), (1, np.float32(-1.0))):
        c.info.seeds_chunk_offset = np.uint32(0)
        prm = c.params("INTEGRATE_TRAJECTORY", sign)
        ot, on, ol, _ = O.integrate_trajectory(prm, n, c.seeds, c.mask, c.uv, integrator=integrator)
        assert np.array_equal(tr.data.traj_nsteps_array[:, d], on)
        assert np.array_equal(tr.data.traj_length_array[:, d].view(np.uint32), ol.view(np.uint32))
        for k in range(n):
            assert np.array_equal(tr.data.streamline_arrays_list[d][k], ot[k, :on[k]])
    ref_stats = compute_stats(tr.data.traj_length_array, tr.data.traj_nsteps_array, c.info.pixel_size)
    assert np.array_equal(tr.data.traj_stats_df.values, ref_stats.values)


def test_fields_stage_raw_and_postprocessed():
    c = Case(nx=56, ny=60, seed=82, density=2, step=0.25, max_length=60.0, n_traj_seeds=200)
    tr = Trajectories(0, 0, info=c.info, data=_data(c))
    tr.integrate()
    stats = tr.data.traj_stats_df
    c2 = Case(nx=56, ny=60, seed=82, density=2, step=0.25, max_length=60.0)
    f = Fields(0, 0, info=c2.info, data=_data(c2, stats))
    seeds, ns, npad = create_seeds(c2.mask, 2, 32)
    f.data.seed_point_array = seeds
    c2.info.n_seed_points, c2.info.n_padded_seed_points = ns, npad
    f.gpu_integrate()
    nxp, nyp = c2.mask.shape
    raw_slc = f.data.slc_array.copy()
    for d, sign in ((0, 1.0), (1, -1.0)):
        prm = c2.params("INTEGRATE_FIELDS", sign)
        oslc, oslt, osteps, _ = O.integrate_fields(prm, seeds, c2.mask, c2.uv, n_threads=4)
        assert np.array_equal(raw_slc[:, :, d], oslc.astype(np.uint32).reshape(nxp, nyp))
        assert f.n_steps[d] == osteps
    # full integrate(): the reference's post-processing on the same raw sums
    c3 = Case(nx=56, ny=60, seed=82, density=2, step=0.25, max_length=60.0)
    f2 = Fields(0, 0, info=c3.info, data=_data(c3, stats))
    f2.integrate()
    assert f2.data.slc_array.shape == (nxp, nyp, 2) and f2.data.slt_array.dtype == np.float32
    expect_slc = np.sqrt(2.0) * np.power(raw_slc / 4, 2 / 3)
    assert np.array_equal(f2.data.slc_array, expect_slc)
    assert np.isfinite(f2.data.sla_array).all()


def _host_finish(data, info, stats):
    """The reference's integrate() post-processing (fields.py:146-167) on the
    raw arrays gpu_integrate() leaves, in NumPy."""
    dds = stats["ds"]["downstream", "mean"]
    uds = stats["ds"]["upstream", "mean"]
    slt = data.slt_array.copy()
    slt[:, :, 0] = slt[:, :, 0] * (dds / info.pixel_size)
    slt[:, :, 1] = slt[:, :, 1] * (uds / info.pixel_size)
    slt = np.sqrt(slt)
    slc = np.sqrt(2.0) * np.power(data.slc_array / info.subpixel_seed_point_density ** 2, 2 / 3)
    return slc, slt, data.sla_array.copy()


@pytest.mark.parametrize("density,exact", [(2, False), (3, False), (2, True)])
def test_fields_device_finish_matches_host(density, exact):
    """integrate() finishes the fields on the GPU; the arrays equal the
    reference's host post-processing of the same raw sums bit for bit."""
    kw = dict(nx=70, ny=52, seed=83, density=density, step=0.25, max_length=60.0)
    ct = Case(n_traj_seeds=200, **kw)
    tr = Trajectories(0, 0, info=ct.info, data=_data(ct))
    tr.integrate()
    stats = tr.data.traj_stats_df
    a = Case(**kw)
    fa = Fields(0, 0, info=a.info, data=_data(a, stats), exact=exact)
    fa.integrate()
    b = Case(**kw)
    fb = Fields(0, 0, info=b.info, data=_data(b, stats), exact=exact)
    seeds, ns, npad = create_seeds(b.mask, 2, b.info.n_work_items)
    fb.data.seed_point_array = seeds
    b.info.n_seed_points, b.info.n_padded_seed_points = ns, npad
    fb.gpu_integrate()
    slc, slt, sla = _host_finish(fb.data, b.info, stats)
    assert fa.data.slc_array.dtype == np.float64 and fa.data.slt_array.dtype == np.float32
    assert np.array_equal(fa.data.slc_array, slc)
    assert np.array_equal(fa.data.slt_array.view(np.uint32), slt.view(np.uint32))
    assert np.array_equal(fa.data.sla_array.view(np.uint32), sla.view(np.uint32))
    # without the table the kernel's own pow stays within 2 ulp
    c = Case(**kw)
    fc = Fields(0, 0, info=c.info, data=_data(c, stats), exact=exact)
    fc.SLC_TABLE_MAX = 0
    fc.integrate()
    assert np.allclose(fc.data.slc_array, slc, rtol=4.5e-16, atol=0.0)
    assert np.array_equal(fc.data.slt_array, slt)


def test_trace_stage_on_a_cropped_region():
    """Trace.do() with real kernels: the fields of the unmasked bounding box
    (Fields run directly on the same crop), zero outside it, slc truncated to
    uint32; trajectory seeds inside the box."""
    import types

    from slm_b200.trace import Trace
    from slm_b200.useful import Info, default_parameters, get_bbox
    c = Case(nx=60, ny=52, seed=83, density=2, step=0.25, max_length=50.0, n_traj_seeds=100)
    pad = 2
    mask = c.mask.copy()
    mask[:pad + 9, :] = True  # a masked band: the crop is smaller than the ROI
    mask[:, -(pad + 6):] = True
    d = default_parameters()
    state = types.SimpleNamespace(**vars(d.state))
    state.merge_active_masks = lambda: mask.copy()
    params = {"trace": dict(vars(d.trace), subpixel_seed_point_density=2, integrator_step_factor=0.25,
                            max_length=50.0, n_trajectory_seed_points=100)}
    geodata = types.SimpleNamespace(roi_nx=60, roi_ny=52, pad_width=pad, roi_pixel_size=1.0)
    t = Trace(state, params, geodata, types.SimpleNamespace(uv_array=c.uv))
    t.do()
    bbox, bnx, bny = get_bbox(~mask)
    b = Data(info=None, bbox=bbox, pad=pad, mask_array=mask, uv_array=c.uv).bounds_slx
    tr = types.SimpleNamespace(**params["trace"])
    info = Info(state, tr, 1.0)
    info.set_xy(bnx, bny, pad)
    data = Data(info=info, bbox=bbox, pad=pad, mask_array=mask, uv_array=c.uv,
                mapping_array=np.zeros(mask.shape, np.uint32), traj_stats_df=t.traj_stats_df)
    f = Fields(0, 0, info=info, data=data)
    f.integrate()
    assert np.array_equal(t.slc_array[b], f.data.slc_array.astype(np.uint32))
    assert np.array_equal(t.slt_array[b], f.data.slt_array)
    outside = np.ones(mask.shape, bool)
    outside[b[:2]] = False
    assert not t.slc_array[outside].any() and t.slc_array[b].any()
    x, y = t.seed_point_array[:, 0] + pad, t.seed_point_array[:, 1] + pad
    assert (x >= bbox[0]).all() and (x <= bbox[1]).all() and (y >= bbox[2]).all() and (y <= bbox[3]).all()


@pytest.mark.parametrize("trace", [False, True])
def test_fields_prepared_work_is_the_same(trace):
    """Fields.prepare (the seed list, and with trace both passes, on a worker
    thread and a side stream while the caller traces trajectories) gives the
    same seed list, fields, step counts and generator state as integrate()
    alone."""
    c = Case(nx=70, ny=66, seed=83, density=2, step=0.25, max_length=60.0, n_traj_seeds=200)
    tr = Trajectories(0, 0, info=c.info, data=_data(c))
    tr.integrate()
    stats = tr.data.traj_stats_df
    out = []
    for prepared in (False, True):
        cc = Case(nx=70, ny=66, seed=83, density=2, step=0.25, max_length=60.0)
        f = Fields(0, 0, info=cc.info, data=_data(cc))
        if prepared:
            f.prepare(trace=trace)
            ct = Case(nx=70, ny=66, seed=83, n_traj_seeds=200)
            Trajectories(0, 0, info=ct.info, data=_data(ct)).integrate()  # runs meanwhile
        f.data.traj_stats_df = stats
        np.random.seed(777)
        f.integrate()
        out.append((f.data.seed_point_array, f.data.slc_array, f.data.slt_array, f.data.sla_array,
                    np.random.get_state(), list(f.n_steps)))
    a, b = out
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2].view(np.uint32), b[2].view(np.uint32))
    assert np.array_equal(a[3].view(np.uint32), b[3].view(np.uint32))
    assert np.array_equal(a[4][1], b[4][1]) and a[4][2] == b[4][2]
    assert a[5] == b[5]
