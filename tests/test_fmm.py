"""Fast-marching lengths on the CPU: the oracle's restatement of the method
(exact cases), its per-subsegment solver against the reference's own phi
construction, and the call-site rules of ``slm_b200.fmm.fmm_lengths`` with a
stand-in solver."""
import numpy as np
import pytest

import eikonal as E
from slm_b200 import fmm


def test_straight_contours_are_exact():
    """Second order marches exactly away from a straight contour, across it
    too (the frozen value on the other side enters negated)."""
    phi = np.ones((11, 7))
    phi[5, :] = -1
    d = E.distance(phi, dx=2.0)
    assert np.array_equal(d.data[:, 3], [9.0, 7.0, 5.0, 3.0, 1.0, -1.0, 1.0, 3.0, 5.0, 7.0, 9.0])
    phi = np.ones((5, 9))
    phi[:, 3:5] = -1
    d = E.distance(phi).data
    assert np.array_equal(d[2], [2.5, 1.5, 0.5, -0.5, -0.5, 0.5, 1.5, 2.5, 3.5])


def test_first_order_and_masks():
    phi = np.ones((9, 9))
    phi[4, 4] = -1
    d1 = E.distance(phi, order=1).data
    # first order along the axes: 0.5 then steps of 1
    assert np.array_equal(d1[4, 5:], [0.5, 1.5, 2.5, 3.5])
    # a masked wall cuts the domain: the far side is not reached
    m = np.ma.MaskedArray(phi, mask=np.zeros_like(phi, bool))
    m.mask[:, 6] = True
    out = E.distance(m)
    assert out.mask[:, 6:].all() and not out.mask[:, :6].any()


def test_no_zero_contour_raises():
    with pytest.raises(ValueError):
        E.distance(np.ones((4, 4)))


def test_symmetric_and_increasing_from_a_point():
    phi = np.ones((15, 15))
    phi[7, 7] = -1
    d, reached = E.distance_unit(phi, np.ones_like(phi, bool))
    assert reached.all()
    assert np.array_equal(d, d.T) and np.array_equal(d, d[::-1, :])
    r = np.hypot(*np.mgrid[-7:8, -7:8])
    far = r > 3
    assert np.abs(d[far] - (r[far] - 0.5)).max() < 0.35


def _case(seed=1, nx=40, ny=36):
    """Labels in blocks (both signs) with thin-channel pixels along lines."""
    rng = np.random.default_rng(seed)
    label = np.zeros((nx, ny), np.int32)
    k = 1
    for x0 in range(0, nx, 10):
        for y0 in range(0, ny, 9):
            label[x0:x0 + 10, y0:y0 + 9] = k * (1 if rng.random() < 0.5 else -1)
            k += 1
    flags = np.zeros((nx, ny), np.uint32)
    thin = np.uint32(1 << 5)
    for x in range(nx):
        y = (x * 3 + seed) % ny
        flags[x, y] |= thin
    flags[rng.random((nx, ny)) < 0.03] |= thin
    flags[rng.random((nx, ny)) < 0.2] |= np.uint32(1 << 2)  # other flags do not matter
    return label, flags, int(thin)


def test_oracle_solver_matches_reference_construction():
    """The solver's per-subsegment phi and mean are those the reference's
    fmm_lengths builds (mapping.py:841-880) given the same distance."""
    from scipy.ndimage import binary_dilation, generate_binary_structure
    label, flags, thin = _case()
    keys = np.unique(np.abs(label[label != 0]))
    sums, counts, n_phi, n_chan, status, per = E.solve_problems(label, flags, thin, keys, 2.0, 2, fields=True)
    for i, s in enumerate(keys):
        phi_bool = np.abs(label) == s
        dil = binary_dilation(phi_bool, structure=generate_binary_structure(2, 1), iterations=1)
        phi = dil.astype(np.float32)
        chan = ((flags & thin) == thin) & (np.abs(label) == s)
        phi[chan] = -1
        pm = np.ma.MaskedArray(phi, ~dil)
        assert n_phi[i] == phi_bool.sum() and n_chan[i] == pm[pm == -1].size
        if n_chan[i] == 0:
            assert status[i] == 1
            continue
        d = E.distance(pm, dx=2.0)
        assert status[i] == 0
        assert np.array_equal(np.ma.filled(d, 0.0), per[i][0])
        assert np.isclose(sums[i] / counts[i], np.mean(d), rtol=1e-12)


def test_call_site_rules():
    """Ratio test (> 4 pixels per channel pixel), doubled mean truncated into
    int32, skipped problems left at 0, both signs of a label sharing one
    problem."""
    calls = []

    def solver(label, flags, thin_bit, keys, dx, order):
        calls.append(list(keys))
        # keys 2, 3, 5, 7: ok (ratio 5), ratio exactly 4, no contour, no channel
        table = {2: (7.9, 2, 10, 2, 0), 3: (7.9, 2, 8, 2, 0), 5: (1.0, 1, 10, 1, 2), 7: (0.0, 0, 10, 0, 1)}
        rows = [table[int(k)] for k in keys]
        return tuple(np.array([r[j] for r in rows]) for j in range(5))

    hsl = fmm.fmm_lengths(None, None, 1, [-7, -2, 2, 3, 5], 1.0, solver=solver)
    assert calls == [[2, 3, 5, 7]]
    assert hsl.dtype == np.int32
    # 7.9 / 2 * 2 = 7.9 -> 7 (truncated); ratio 8/2 = 4 is not > 4
    assert hsl.tolist() == [0, 7, 7, 0, 0]
    assert fmm.fmm_lengths(None, None, 1, [], 1.0, solver=solver).size == 0
