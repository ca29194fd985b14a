"""The device seed list (slm_create_seeds_device) against the host one.

slm_create_seeds is pinned to NumPy's own argwhere + legacy shuffle
(tests/test_seeds.py); the device list must hold the same rows in the same
order and leave the same generator state, including the edge cases: no
unmasked pixel, one, two, a truncated list, and grids up to 4100^2 (16.6 M
rows: the swaps go to the device in chunks of 4 M as they are drawn).
"""
import ctypes

import numpy as np
import pytest
import torch

from slm_b200 import _lib
from slm_b200 import useful as U

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


def _host(mask, pad, do_shuffle, seed):
    rows, _, _ = U.create_seeds(mask, pad, 64, do_shuffle=do_shuffle, rng_seed=seed)
    return rows, np.random.get_state()


def _device(mask, pad, do_shuffle, seed, n_seed_points=None):
    t, n, npad = U.create_seeds_device(mask, pad, 64, DEV, n_seed_points=n_seed_points, do_shuffle=do_shuffle,
                                       rng_seed=seed)
    torch.cuda.synchronize()
    return t.cpu().numpy(), n, npad, np.random.get_state()


def _mask(shape, frac, seed):
    m = np.random.default_rng(seed).random(shape) < frac
    m[:2], m[-2:], m[:, :2], m[:, -2:] = True, True, True, True
    return m


@pytest.mark.parametrize("shape,frac,seed,do_shuffle", [
    ((9, 11), 1.0, 1, True),          # every pixel masked: no rows
    ((9, 11), 0.0, 2, True),
    ((5, 5), 0.0, 3, True),           # one unmasked pixel
    ((5, 6), 0.0, 4, True),           # two
    ((37, 29), 0.3, 5, True),
    ((37, 29), 0.3, 6, False),        # no shuffle: argwhere order
    ((300, 257), 0.1, 7, True),
    ((1030, 1030), 0.02, 8, True),
    ((2052, 2052), 0.01, 9, True),
    ((4100, 4100), 0.01, 11, True),   # 16.6 M rows: four chunks of swaps, drawn while earlier ones run
])
def test_device_seeds_equal_host_seeds(shape, frac, seed, do_shuffle):
    mask = _mask(shape, frac, seed)
    want, want_state = _host(mask, 2, do_shuffle, seed)
    np.random.seed(12345)  # the device call must set the state itself
    got, n, npad, got_state = _device(mask, 2, do_shuffle, seed)
    assert n == want.shape[0]
    assert got.shape == want.shape and np.array_equal(got, want)
    if do_shuffle:
        assert np.array_equal(got_state[1], want_state[1]) and got_state[2] == want_state[2]
    assert npad % 64 == 0 and npad >= n


def test_device_seeds_truncated_list():
    mask = _mask((200, 180), 0.05, 10)
    want, n_want, npad_want = U.create_seeds(mask, 2, 32, n_seed_points=1000, do_shuffle=True, rng_seed=1)
    t, n, npad = U.create_seeds_device(mask, 2, 32, DEV, n_seed_points=1000, do_shuffle=True, rng_seed=1)
    assert (n, npad) == (n_want, npad_want)
    assert np.array_equal(t.cpu().numpy(), want)


def test_device_seeds_reject_small_buffers():
    L = _lib.load()
    mask = torch.zeros((20, 20), dtype=torch.uint8, device=DEV)
    n = ctypes.c_uint64(0)
    ws = torch.empty(int(L.slm_create_seeds_device_workspace(400)), dtype=torch.uint8, device=DEV)
    out = torch.empty((100, 2), dtype=torch.float32, device=DEV)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.slm_create_seeds_device(_lib.ptr(mask), 20, 20, 2, 1, 1, _lib.ptr(out), 100, ctypes.byref(n), None,
                                   _lib.ptr(ws), ws.numel(), s)
    assert rc == _lib.SLM_ERR_CAPACITY and n.value == 400
    rc = L.slm_create_seeds_device(_lib.ptr(mask), 20, 20, 2, 1, 1, _lib.ptr(out), 400, ctypes.byref(n), None,
                                   _lib.ptr(ws), ws.numel() - 1, s)
    assert rc == _lib.SLM_ERR_ARGS
