"""The reference's IndianCreek Test#2 job on its real DTM through the GPU
stages: Preprocess (the conditioned uv, bit-exact with the oracle and the
notebook's 62 blockages), Trace (Trajectories + Fields; the notebook's step
counts exactly, l and ds within tests/indiancreek.py's tolerances), and the
raw field sums of the job's 15930 seeds (d=3, RK2) bit-exact with the
oracle, and with the reference's own kernel where it was built."""
import os
import types

import numpy as np
import pytest

import dtm_preprocess as DP
import indiancreek as IC
import oracle as O
from slm_b200.fields import Fields
from slm_b200.preprocess import conditioned_gradient_vector_field
from slm_b200.trace import Trace
from slm_b200.useful import create_seeds

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def job():
    roi, basin, pixel_size = IC.load()
    pre = conditioned_gradient_vector_field(roi, pixel_size, IC.PAD)
    mask = IC.masks(roi, basin, pre.uv_mask_array)
    return roi, pre, mask, pixel_size


def test_preprocess_on_gpu(job):
    roi, pre, mask, pixel_size = job
    ref = DP.conditioned_uv(roi, pixel_size, IC.PAD)
    assert np.array_equal(pre.uv_array.view(np.uint32), ref["uv_array"].view(np.uint32))
    assert int((pre.blockages_array != 0).sum()) == IC.N_BLOCKAGES
    assert int((~mask).sum()) == IC.N_FIELD_SEEDS


def test_trace_stage_matches_the_notebook(job):
    _, pre, mask, pixel_size = job
    geodata = types.SimpleNamespace(roi_nx=200, roi_ny=200, pad_width=IC.PAD, roi_pixel_size=pixel_size)
    t = Trace(IC.state_for(mask), {"trace": {}}, geodata, types.SimpleNamespace(uv_array=pre.uv_array))
    t.do()
    df = t.traj_stats_df
    got = t.streamline_arrays_list
    n = np.stack([[len(a) for a in got[0]], [len(a) for a in got[1]]], 1)
    IC.check_stats(n, got)
    assert df["n"]["downstream", "max"] == 563 and df["n"]["upstream", "max"] == 2000
    assert t.slc_array.shape == (204, 204, 2) and t.slc_array.any()


def test_field_sums_bit_exact(job):
    _, pre, mask, pixel_size = job
    info, data = IC.trace_inputs(mask, pre.uv_array, pixel_size)
    seeds, ns, npad = create_seeds(data.mask_array, info.pad_width, info.n_work_items)
    assert ns == IC.N_FIELD_SEEDS
    info.n_seed_points, info.n_padded_seed_points = ns, npad
    data.seed_point_array = seeds
    f = Fields(0, 0, info=info, data=data)
    f.gpu_integrate()
    nxp, nyp = data.mask_array.shape
    for col, sign in enumerate((1.0, -1.0)):
        prm = IC.field_params(info, sign)
        oslc, oslt, osteps, _ = O.integrate_fields(prm, seeds, data.mask_array, data.uv_array, 2,
                                                   n_threads=os.cpu_count() or 1)
        assert np.array_equal(f.data.slc_array[:, :, col], oslc.astype(np.uint32).reshape(nxp, nyp))
        assert f.n_steps[col] == osteps
        if O.ref_available("integrate_fields"):
            rslc, rslt = O.ref_integrate_fields(prm, seeds, data.mask_array, data.uv_array,
                                                n_threads=os.cpu_count() or 1)
            assert np.array_equal(f.data.slc_array[:, :, col], rslc.reshape(nxp, nyp))
            assert np.array_equal((oslt & 0xFFFFFFFF).astype(np.uint32), rslt)
