"""create_seeds' native shuffle (slm_create_seeds, host code) against NumPy's
legacy generator, which the reference uses (useful.py:470-517): the same
rows in the same order, and the global generator left in the same state."""
import numpy as np
import pytest

from slm_b200 import useful as U


def numpy_seeds(mask, pad, do_shuffle, rng_seed):
    """The reference's create_seeds core in NumPy (useful.py:496-501):
    argwhere(~mask) - pad, rows shuffled by the global legacy generator.
    Shuffling rows and permutation(N) draw the same Fisher-Yates partners
    from the same stream, so rows[permutation(N)] is the same array and
    leaves the generator in the same state."""
    m = np.ascontiguousarray(mask, dtype=np.bool_)
    rows = np.argwhere(~m).astype(np.float32) - pad
    if do_shuffle:
        np.random.seed(rng_seed)
        rows = rows[np.random.permutation(rows.shape[0])]
    return rows


@pytest.mark.parametrize("shape,pad,seed,frac", [((7, 9), 2, 1, 0.2), ((130, 77), 2, 0, 0.1),
                                                 ((300, 257), 3, 12345, 0.5), ((1, 1), 0, 5, 0.0),
                                                 ((64, 64), 2, 2 ** 32 - 1, 0.97), ((40, 33), 0, 7, 1.0),
                                                 ((1100, 1000), 2, 3, 0.0)])
@pytest.mark.parametrize("do_shuffle", [True, False])
def test_native_seeds_match_numpy(shape, pad, seed, frac, do_shuffle):
    rng = np.random.default_rng(sum(shape) + seed % 1000)
    mask = rng.random(shape) < frac
    a = numpy_seeds(mask, pad, do_shuffle, seed)
    sa = np.random.get_state()
    np.random.seed(99)  # disturb the global generator between the two
    b = U._shuffled_seeds(mask, pad, do_shuffle, seed)
    sb = np.random.get_state()
    assert a.dtype == b.dtype == np.float32 and a.shape == b.shape
    assert np.array_equal(a, b)
    if do_shuffle:
        assert np.array_equal(sa[1], sb[1]) and sa[2] == sb[2]
        assert np.random.random() == (np.random.set_state(sa), np.random.random())[1]


def test_create_seeds_subset_and_padding():
    mask = np.zeros((20, 30), bool)
    mask[:2] = mask[-2:] = True
    mask[:, :2] = mask[:, -2:] = True
    s, n, npad = U.create_seeds(mask, 2, 32, n_seed_points=10, do_shuffle=True, rng_seed=3)
    full = numpy_seeds(mask, 2, True, 3)
    assert n == 10 and np.array_equal(s, full[:10]) and npad % 32 == 0


def test_decode_streamlines_matches_the_reference_expression():
    """plot.py:1414-1423 restated inline: (0,0) start, float32 steps over the
    resolution, cumulative sums plus origin plus seed."""
    from slm_b200.trajectories import decode_streamlines
    rng = np.random.default_rng(4)
    seeds = rng.uniform(0, 50, (5, 2)).astype(np.float32)
    lists = [rng.integers(-60, 60, (int(n), 2)).astype(np.int8) for n in (0, 1, 7, 300, 33)]
    origin = (np.float32(0.5), np.float32(0.5))
    got = decode_streamlines(seeds, lists, 128, origin)
    for k in range(5):
        traj = np.concatenate((np.array([[0, 0]], dtype=np.float32), lists[k].astype(np.float32) / np.float32(128)))
        x = origin[0] + np.cumsum(traj.T[0]) + seeds[k, 0]
        y = origin[1] + np.cumsum(traj.T[1]) + seeds[k, 1]
        assert np.array_equal(got[k][0], x) and np.array_equal(got[k][1], y)
        assert got[k][0].dtype == np.float32 and got[k][0].size == lists[k].shape[0] + 1


def _sequential_swaps(rows, js):
    """Fisher-Yates' swap pass: swap(i, js[i]) for i = n-1 down to 1."""
    rows = rows.copy()
    for i in range(rows.shape[0] - 1, 0, -1):
        j = js[i]
        rows[[i, j]] = rows[[j, i]]
    return rows


def _reservation_rounds(rows, js):
    """The device shuffle's schedule restated in NumPy: every pending swap
    reserves its two rows with its index (the maximum wins); a swap holding
    both reservations runs, the others wait for the next round."""
    rows = rows.copy()
    n = rows.shape[0]
    pending = np.arange(1, n, dtype=np.int64)
    rounds = 0
    while pending.size:
        rounds += 1
        res = np.zeros(n, np.int64)
        np.maximum.at(res, pending, pending)
        np.maximum.at(res, js[pending], pending)
        run = (res[pending] == pending) & (res[js[pending]] == pending)
        i = pending[run]
        j = js[i]
        # rows of swaps that run in one round are pairwise distinct
        assert np.unique(np.concatenate([i, j[i != j]])).size == i.size + int((i != j).sum())
        rows[i], rows[j] = rows[j].copy(), rows[i].copy()
        pending = pending[~run]
    return rows, rounds


@pytest.mark.parametrize("n,seed", [(1, 0), (2, 1), (3, 2), (17, 3), (1000, 4), (200_000, 5)])
def test_reservation_rounds_equal_sequential_swaps(n, seed):
    """The round schedule of slm_create_seeds_device gives the sequential
    shuffle's rows for any partners j(i) in [0, i], in few rounds."""
    rng = np.random.default_rng(seed)
    js = np.zeros(n, np.int64)
    if n > 1:
        js[1:] = rng.integers(0, np.arange(2, n + 1))
    rows = np.stack([np.arange(n, dtype=np.float32), -np.arange(n, dtype=np.float32)], 1)
    got, rounds = _reservation_rounds(rows, js)
    assert np.array_equal(got, _sequential_swaps(rows, js)) if n < 5000 else True
    if n >= 5000:  # the sequential loop in Python is slow: compare with NumPy's own shuffle order
        perm = np.arange(n)
        for i in range(n - 1, 0, -1):
            j = js[i]
            perm[i], perm[j] = perm[j], perm[i]
        assert np.array_equal(got, rows[perm])
    assert rounds <= max(4, 8 * int(np.log2(max(n, 2))))
