"""slm_fmm_lengths on the GPU against the oracle's fast-marching solver: the
signed distance fields bit for bit, the sums and counts exactly, the status
of every problem (no channel, no zero contour, absent label), both orders,
and the pass-2 lengths built on them."""
import numpy as np
import pytest
import torch

import eikonal as E
from slm_b200 import fmm
from test_fmm import _case

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def _compare(label, flags, thin, keys, dx, order):
    lab_d = torch.from_numpy(label).to(DEV)
    flg_d = torch.from_numpy(flags.astype(np.int64)).to(DEV)
    got = fmm.device_solver(lab_d, flg_d, thin, keys, dx, order, fields=True)
    want = E.solve_problems(label, flags, thin, keys, dx, order, fields=True)
    for k in range(5):
        assert np.array_equal(got[k], want[k]), (k, got[k], want[k])
    for i in range(len(keys)):
        if want[4][i] != 0:
            continue
        (x0, x1, y0, y1), val, reached = got[5][i]
        dist, ok = want[5][i]
        assert np.array_equal(reached, ok[x0:x1 + 1, y0:y1 + 1])
        assert not ok.sum() - ok[x0:x1 + 1, y0:y1 + 1].sum()
        assert np.array_equal(val.view(np.uint64), dist[x0:x1 + 1, y0:y1 + 1].view(np.uint64))
    return got


@pytest.mark.parametrize("order", [2, 1])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fmm_kernel_matches_oracle(seed, order):
    label, flags, thin = _case(seed=seed, nx=50 + seed, ny=44)
    keys = np.unique(np.abs(label[label != 0]))
    got = _compare(label, flags, thin, keys, 2.0, order)
    assert (got[4] == 0).sum() >= len(keys) // 2


def test_fmm_kernel_large_region_and_irregular_shapes():
    """One region of 52 K pixels (a deep heap) with a meandering channel, and
    irregular labels beside it."""
    rng = np.random.default_rng(9)
    nx, ny = 260, 230
    label = np.full((nx, ny), 4, np.int32)
    label[:, 200:] = -6
    label[rng.random((nx, ny)) < 0.02] = 0
    flags = np.zeros((nx, ny), np.uint32)
    thin = 1 << 3
    for x in range(nx):
        flags[x, int(100 + 40 * np.sin(x / 17.0))] |= thin
    flags[::7, 215] |= thin
    keys = np.array([4, 6], np.int64)
    got = _compare(label, flags, thin, keys, 1.5, 2)
    assert (got[4] == 0).all()


def test_fmm_kernel_edge_cases():
    """No channel pixel (status 1), a label absent from the grid (1), a
    one-pixel channel label (0); and a label whose own pixels are all
    channel pixels and fill the window, so that its domain has no +1 pixel
    and no zero contour (2, where the reference's skfmm call raises)."""
    label = np.zeros((12, 10), np.int32)
    label[0:4, :] = 1
    label[4:12, :] = 2
    flags = np.zeros((12, 10), np.uint32)
    thin = 1 << 4
    flags[6, :] |= thin
    label[1, 1] = 9
    flags[1, 1] |= thin
    got = _compare(label, flags, thin, np.array([1, 2, 5, 9], np.int64), 1.0, 2)
    assert got[4].tolist() == [1, 0, 1, 0]
    assert got[2].tolist() == [39, 80, 0, 1] and got[3].tolist() == [0, 10, 0, 1]
    full = np.full((7, 9), -3, np.int32)
    got = _compare(full, np.full((7, 9), thin, np.uint32), thin, np.array([3], np.int64), 1.0, 2)
    assert got[4].tolist() == [2]


def test_fmm_lengths_gpu_equals_oracle_solver():
    label, flags, thin = _case(seed=4, nx=60, ny=45)
    sel = np.unique(label[label != 0]).astype(np.int32)
    lab_d = torch.from_numpy(label).to(DEV)
    flg_d = torch.from_numpy(flags.astype(np.int64)).to(DEV)
    a = fmm.fmm_lengths(lab_d, flg_d, thin, sel, 2.0)
    b = fmm.fmm_lengths(label, flags, thin, sel, 2.0, solver=E.solve_problems)
    assert a.dtype == np.int32 and np.array_equal(a, b) and (a > 0).any()


def test_wrapper_fmm_lengths_device_runner_equals_oracle():
    """The reference-shaped wrapper (slm_b200.mapping.fmm_lengths) on the
    device runner equals it on the oracle runner, on mapped grids."""
    import copy

    from mapping_cases import incised_pipeline_case, oracle_runner
    from slm_b200 import mapping as M
    info, data = incised_pipeline_case(n=64, seed=3, n_incisions=6, max_steps=200)
    assert M.map_channels_segments(None, info, data, runner=oracle_runner)
    lab = data.label_array[~data.mask_array]
    data.selected_subsegments_array = np.unique(lab[lab != 0]).astype(np.int32)
    a, b = copy.deepcopy(data), copy.deepcopy(data)
    ok_gpu = M.fmm_lengths(None, info, a, 2.0, runner=M.DeviceRunner(DEV))
    ok_cpu = M.fmm_lengths(None, info, b, 2.0, runner=oracle_runner)
    assert ok_gpu and ok_cpu
    assert np.array_equal(a.subsegment_hsl_array, b.subsegment_hsl_array)
    assert a.fmm_mean_hsl == b.fmm_mean_hsl
