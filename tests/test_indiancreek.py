"""The reference's IndianCreek Test#2 job on its real DTM, through the oracle
(CPU): the preprocess's blockage count, the field seed count, and the
trajectory statistics its notebook recorded (tests/indiancreek.py)."""
import os

import numpy as np
import pytest

import dtm_preprocess as DP  # noqa: E402
import indiancreek as IC
import oracle as O
from slm_b200.params import kernel_params
from slm_b200.useful import create_seeds


@pytest.fixture(scope="module")
def job():
    roi, basin, pixel_size = IC.load()
    pre = DP.conditioned_uv(roi, pixel_size, IC.PAD)
    mask = IC.masks(roi, basin, pre["uv_mask_array"])
    return roi, pre, mask, pixel_size


def test_fixture_is_the_reference_data(reference_dir, tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_indiancreek_golden", os.path.join(os.path.dirname(IC.GOLDEN), "make_indiancreek_golden.py"))
    G = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(G)
    out = G.make(reference_dir, str(tmp_path / "ic.npz"))
    a, b = np.load(out), np.load(IC.GOLDEN)
    assert np.array_equal(a["roi"], b["roi"], equal_nan=True)
    assert np.array_equal(a["basin_mask"], b["basin_mask"])


def test_preprocess_and_seed_counts(job):
    roi, pre, mask, _ = job
    assert roi.shape == (200, 200)
    assert int((pre["blockages_array"] != 0).sum()) == IC.N_BLOCKAGES
    assert int((~mask).sum()) == IC.N_FIELD_SEEDS


def test_trajectory_statistics_match_the_notebook(job):
    _, pre, mask, pixel_size = job
    info, data = IC.trace_inputs(mask, pre["uv_array"], pixel_size)
    seeds, n, _ = create_seeds(data.mask_array, info.pad_width, info.n_work_items,
                               n_seed_points=info.n_trajectory_seed_points, do_shuffle=True, rng_seed=1)
    info.n_seed_points = n
    nsteps = np.zeros((n, 2), np.uint16)
    lists = [[], []]
    for col, sign in enumerate((1.0, -1.0)):
        prm = kernel_params(info, "INTEGRATE_TRAJECTORY", np.float32(sign))
        traj, ns, ln, _ = O.integrate_trajectory(prm, n, seeds, data.mask_array, data.uv_array, 2,
                                                 n_threads=os.cpu_count() or 1)
        nsteps[:, col] = ns
        lists[col] = [traj[k, :ns[k]] for k in range(n)]
        if O.ref_available("integrate_trajectory"):
            rt, rns, rln = O.ref_integrate_trajectory(prm, n, seeds, data.mask_array, data.uv_array)
            assert np.array_equal(rns, ns) and np.array_equal(rln.view(np.uint32), ln.view(np.uint32))
    IC.check_stats(nsteps, lists)
