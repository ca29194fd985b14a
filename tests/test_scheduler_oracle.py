"""CPU checks of the learned length scheduler's oracle and host logic:
bfloat16 rounding, the analytic gradient against finite differences, the
patch layout, and the makespan model used to score seed orders."""
import numpy as np
import torch

import length_model as LM
from slm_b200 import scheduler as S


def _weights(seed=0, scale=1.0):
    p = S.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    for k in p:
        if k.startswith("b"):
            p[k] = (rng.standard_normal(p[k].shape) * 0.1).astype(np.float32)
        p[k] = p[k] * scale
    return p


def test_bf16_matches_torch():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.standard_normal(10000).astype(np.float32) * 10.0 ** rng.integers(-6, 6, 10000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 65504.0, 3.0e38], np.float32)])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(LM.bf16(x), ref)
    assert np.array_equal(S.bf16_round(torch.from_numpy(x)).numpy(), ref)


def test_rearrange_adjoint():
    rng = np.random.default_rng(2)
    a1 = rng.standard_normal((3, 16, 32))
    dx2 = rng.standard_normal((3, 4, 128))
    lhs = (LM._rearrange(a1) * dx2).sum()
    rhs = (a1 * LM._rearrange_back(dx2)).sum()
    assert abs(lhs - rhs) < 1e-9 * max(1.0, abs(lhs))
    # every conv1 activation feeds exactly one conv2 input
    assert np.array_equal(np.sort((LM._T2 * 32 + LM._O2).ravel()), np.arange(512))


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = {k: v.astype(np.float64) for k, v in _weights(3).items()}
    x1 = rng.standard_normal((5, 16, 32))
    t = rng.standard_normal((5, 2))
    _, g = LM.loss_and_grad(w, x1, t, rounding=False)
    h = 1e-6
    for name, _ in LM.SHAPES:
        flat = w[name].ravel()
        for i in rng.choice(flat.size, size=min(12, flat.size), replace=False):
            old = flat[i]
            flat[i] = old + h
            lp, _ = LM.loss_and_grad(w, x1, t, rounding=False)
            flat[i] = old - h
            lm, _ = LM.loss_and_grad(w, x1, t, rounding=False)
            flat[i] = old
            fd = (lp - lm) / (2 * h)
            an = g[name].ravel()[i]
            assert abs(fd - an) <= 1e-6 + 1e-5 * abs(fd), (name, i, fd, an)


def test_gather_layout_and_clamp():
    nxp, nyp, pad = 12, 10, 2
    uv = np.zeros((nxp, nyp, 2), np.float32)
    xs, ys = np.meshgrid(np.arange(nxp), np.arange(nyp), indexing="ij")
    uv[:, :, 0] = xs
    uv[:, :, 1] = ys
    seeds = np.array([[3.5, 4.25], [0.0, 0.0]], np.float32)
    x1 = LM.gather(uv, pad, seeds)
    # tile t = 4*ti + tj, cell m = 4*di + dj, feature f = 2*m + c
    for s, (sx, sy) in enumerate(seeds):
        cx, cy = int(sx) + pad, int(sy) + pad
        for t in range(16):
            for m in range(16):
                x = min(max(cx - 8 + 4 * (t // 4) + m // 4, 0), nxp - 1)
                y = min(max(cy - 8 + 4 * (t % 4) + m % 4, 0), nyp - 1)
                assert x1[s, t, 2 * m] == x and x1[s, t, 2 * m + 1] == y


def test_makespan_longest_first_helps():
    rng = np.random.default_rng(4)
    steps = np.minimum(rng.pareto(1.2, 20000) * 40 + 5, 6000).astype(np.int64)
    shuffled = rng.permutation(steps.size)
    longest = np.argsort(-steps, kind="stable")
    lanes = 256
    a = S.makespan(steps, shuffled, lanes)
    b = S.makespan(steps, longest, lanes)
    lower = max(int(steps.max()), int(np.ceil(steps.sum() / lanes)))
    assert lower <= b <= a
    assert S.makespan(steps[:10], np.arange(10), lanes) == int(steps[:10].max())


def test_warp_cost_model():
    steps = np.array([5, 1, 1, 1, 9, 2, 2, 2])
    assert S.warp_cost(steps, np.arange(8), width=4) == 5 + 9
    assert S.warp_cost(steps, np.array([4, 0, 5, 6, 1, 2, 3, 7]), width=4) == 9 + 2
    rng = np.random.default_rng(5)
    st = np.minimum(rng.pareto(1.2, 50000) * 40 + 5, 6000).astype(np.int64)
    assert S.warp_cost(st, np.argsort(-st)) < S.warp_cost(st, rng.permutation(st.size))
    assert S.warp_cost(st[:33], np.arange(33)) == st[:32].max() + st[32]
