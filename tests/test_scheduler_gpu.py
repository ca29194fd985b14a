"""GPU checks of the learned length scheduler: the GEMM / gather / backward
kernels against the NumPy oracle (gradient check), the fused tensor-core
inference against the oracle's forward pass, the ordering kernel, that a
scheduled trace is bit-identical to the plain one, and that a model trained
on one synthetic DTM orders the seeds of another better than the shuffled
default (makespan model of the persistent kernel)."""
import numpy as np
import pytest
import torch

import length_model as LM
from cases import Case
from slm_b200 import kernels, scheduler as S
from slm_b200.params import kernel_params
from slm_b200.workloads import Workload

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _weights(seed):
    p = S.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    for k in p:
        if k.startswith("b"):
            p[k] = (rng.standard_normal(p[k].shape) * 0.1).astype(np.float32)
    return p


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (70, 33, 45), (128, 64, 200), (5, 130, 17), (300, 256, 130),
                                 (4096, 2, 256), (32, 32, 5000)])
def test_gemm_matches_torch(ta, tb, mnk):
    M, N, K = mnk
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((K, M) if ta else (M, K), generator=g).to(DEV)
    B = torch.randn((N, K) if tb else (K, N), generator=g).to(DEV)
    bias = torch.randn(N, generator=g).to(DEV)
    # the tensor cores take A and B as bfloat16: the exact products of the
    # rounded operands, summed in fp32 (tolerance relative to sum |a b|)
    Ar, Br = S.bf16_round(A).double(), S.bf16_round(B).double()
    opA, opB = (Ar.T if ta else Ar), (Br.T if tb else Br)
    ref = opA @ opB + bias.double()
    mag = opA.abs() @ opB.abs()
    m = S.LengthModel(DEV)
    C = torch.empty(M, N, device=DEV)
    Z = torch.empty(M, N, device=DEV)
    m._gemm(ta, tb, M, N, K, A, B, C, Z, bias, relu=1, rnd=1)
    torch.cuda.synchronize()
    tol = 1e-5 * (mag + bias.double().abs()) + 1e-30
    assert torch.all((Z.double() - ref).abs() <= tol)
    assert torch.equal(C, S.bf16_round(torch.relu(Z)))
    C2 = torch.zeros(M, N, device=DEV)
    m._gemm(ta, tb, M, N, K, A, B, C2, split=3)
    torch.cuda.synchronize()
    assert torch.all((C2.double() - (ref - bias.double())).abs() <= 1e-5 * mag + 1e-30)
    m.check_status()


def _uv_grid(seed, nx=40, ny=36, pad=2):
    rng = np.random.default_rng(seed)
    uv = rng.standard_normal((nx + 2 * pad, ny + 2 * pad, 2)).astype(np.float32)
    seeds = np.stack([rng.uniform(0, nx, 300), rng.uniform(0, ny, 300)], 1).astype(np.float32)
    return uv, seeds


def test_gather_exact():
    uv, seeds = _uv_grid(1)
    idx = np.random.default_rng(2).integers(0, seeds.shape[0], 77).astype(np.int32)
    m = S.LengthModel(DEV)
    x1 = m.gather(torch.from_numpy(uv).to(DEV), uv.shape[0], uv.shape[1], 2,
                  torch.from_numpy(seeds).to(DEV), torch.from_numpy(idx).to(DEV), idx.size)
    ref = LM.gather(uv, 2, seeds, idx).reshape(-1, 32)
    assert np.array_equal(x1.cpu().numpy().astype(np.float64), ref)


def test_gradient_check_against_oracle():
    uv, seeds = _uv_grid(3)
    w = _weights(5)
    n = seeds.shape[0]
    t = np.random.default_rng(4).standard_normal((n, 2)).astype(np.float32)
    m = S.LengthModel(DEV, w)
    uv_d, seeds_d = torch.from_numpy(uv).to(DEV), torch.from_numpy(seeds).to(DEV)
    x1 = m.gather(uv_d, uv.shape[0], uv.shape[1], 2, seeds_d, None, n)
    loss = m.loss_and_grad(x1, torch.from_numpy(t).to(DEV), n)
    torch.cuda.synchronize()
    rl, rg = LM.loss_and_grad(w, LM.gather(uv, 2, seeds), t.astype(np.float64))
    assert abs(float(loss.item()) - rl) <= 1e-5 * abs(rl)
    for name, _ in LM.SHAPES:
        got = m.G[name].cpu().numpy().astype(np.float64)
        ref = rg[name].reshape(got.shape)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 2e-4 * scale + 1e-7, name


def test_inference_matches_oracle_forward():
    uv, seeds = _uv_grid(6, 70, 50)
    seeds = np.concatenate([seeds, seeds[:37]])  # n not a multiple of 16
    w = _weights(7)
    m = S.LengthModel(DEV, w)
    uv_d, seeds_d = torch.from_numpy(uv).to(DEV), torch.from_numpy(seeds).to(DEV)
    pred = m.predict(uv_d, uv.shape[0], uv.shape[1], 2, seeds_d, seeds.shape[0])
    x1 = m.gather(uv_d, uv.shape[0], uv.shape[1], 2, seeds_d, None, seeds.shape[0])
    y = m.forward(x1, seeds.shape[0])
    torch.cuda.synchronize()
    ref = LM.predict(w, uv, 2, seeds)
    scale = np.abs(ref).max()
    assert np.abs(pred.cpu().numpy() - ref).max() <= 2e-3 * scale
    assert np.abs(y.cpu().numpy() - ref).max() <= 2e-3 * scale
    # visiting the seeds in another order changes no prediction
    perm = torch.from_numpy(np.random.default_rng(11).permutation(seeds.shape[0]).astype(np.int32)).to(DEV)
    pred2 = m.predict(uv_d, uv.shape[0], uv.shape[1], 2, seeds_d, seeds.shape[0], visit=perm.view(torch.uint32))
    assert torch.equal(pred, pred2)


def test_order_by_prediction():
    rng = np.random.default_rng(8)
    n = 100003
    pred = np.stack([rng.uniform(-1, 9, n), rng.uniform(0, 8, n)], 1).astype(np.float32)
    pred[5, 0] = np.nan
    m = S.LengthModel(DEV)
    pd = torch.from_numpy(pred).to(DEV)
    for col in (0, 1):
        order = m.order(pd, col, 8.0).cpu().numpy().astype(np.int64)
        assert np.array_equal(np.sort(order), np.arange(n))
        v = np.nan_to_num(pred[order, col], nan=-1.0)
        b = np.floor(np.clip(v / 8.0, 0, 1) * (S.N_BINS - 1) + 0.5)
        assert np.all(np.diff(b) <= 0), "bins not longest first"


def test_scheduled_trace_identical_and_steps_recorded():
    c = Case(nx=72, ny=64, seed=51, density=2, step=0.2, max_length=150.0)
    seeds, mask, uv = (torch.from_numpy(c.seeds).to(DEV), torch.from_numpy(c.mask.view(np.uint8)).to(DEV),
                       torch.from_numpy(c.uv).to(DEV))
    for integrator in (2, 4):
        prm = c.params("INTEGRATE_FIELDS", -1.0 if integrator == 4 else 1.0)
        n, dd = int(prm.n_seed_points), int(prm.subpixel_seed_point_density) ** 2
        perm = torch.from_numpy(np.random.default_rng(9).permutation(n).astype(np.int32)).to(DEV)
        out = []
        for schedule, order in (("persistent", None), ("persistent", perm), ("plain", perm)):
            slc = torch.zeros(prm.nxy_padded, dtype=torch.uint64, device=DEV)
            slt = torch.zeros_like(slc)
            work = kernels.workspace(DEV)
            steps = torch.zeros(n * dd, dtype=torch.uint16, device=DEV)
            kernels.integrate_fields(prm, seeds, mask, uv, slc, slt, work, schedule=schedule,
                                     integrator=integrator, order=order.view(torch.uint32) if order is not None else None,
                                     item_steps=steps)
            torch.cuda.synchronize()
            out.append((slc.cpu().numpy(), slt.cpu().numpy(), int(work[1].item()),
                        steps.cpu().numpy().astype(np.int64)))
        base = out[0]
        assert base[3].sum() == base[2]
        p = perm.cpu().numpy().astype(np.int64)
        for o in out[1:]:
            assert np.array_equal(o[0], base[0]) and np.array_equal(o[1], base[1])
            assert o[2] == base[2]
            assert np.array_equal(o[3].reshape(n, dd), base[3].reshape(n, dd)[p])


def _trained_and_eval():
    train, ev = Workload("incised512", seed=21), Workload("incised512", seed=22)
    m = S.LengthModel(DEV, seed=0)

    def dev(wl):
        return (torch.from_numpy(wl.seeds).to(DEV), torch.from_numpy(wl.mask.view(np.uint8)).to(DEV),
                torch.from_numpy(wl.uv).to(DEV))

    def targets(wl):
        seeds, mask, uv = dev(wl)
        cols = []
        for sign in (1.0, -1.0):
            prm = kernel_params(wl.info, "INTEGRATE_FIELDS", sign)
            st = S.record_steps(prm, seeds, mask, uv, integrator=wl.spec.integrator)
            cols.append(st)
        return cols, prm

    (tr_dn, tr_up), prm = targets(train)
    n_tr = int(train.info.n_seed_points)
    d = train.spec.density
    t = torch.stack([S.step_targets(tr_dn, n_tr, d), S.step_targets(tr_up, n_tr, d)], 1).contiguous()
    seeds, _, uv = dev(train)
    hist = m.fit(uv, uv.shape[0], uv.shape[1], 2, seeds, t, steps=1500, batch=4096)
    (ev_dn, ev_up), prm_ev = targets(ev)
    return m, hist, ev, (ev_dn, ev_up), prm_ev, dev(ev)


def test_learned_order_beats_shuffled():
    """Trained on one synthetic DTM, the model's order of another DTM's seeds
    lowers the plain kernel's cost (sum over warps of the longest lane) below
    the shuffled default's, and its predictions rank-correlate with the true
    step counts."""
    m, hist, ev, (ev_dn, ev_up), prm, (seeds, mask, uv) = _trained_and_eval()
    assert np.mean(hist[-20:]) < 0.5 * np.mean(hist[:20])
    n = int(ev.info.n_seed_points)
    dd = ev.spec.density ** 2
    pred = m.predict(uv, uv.shape[0], uv.shape[1], 2, seeds, n)
    for col, st in ((0, ev_dn), (1, ev_up)):
        order = m.order(pred, col, S.log_cap(prm)).cpu().numpy().astype(np.int64)
        steps = st.cpu().numpy().astype(np.int64).reshape(n, dd)
        items = lambda o: (o[:, None] * dd + np.arange(dd)[None, :]).ravel()
        flat = steps.ravel()
        shuffled = S.warp_cost(flat, np.arange(n * dd))
        learned = S.warp_cost(flat, items(order))
        ideal = S.warp_cost(flat, np.argsort(-flat, kind="stable"))
        rho = np.corrcoef(np.argsort(np.argsort(pred[:, col].cpu().numpy())),
                          np.argsort(np.argsort(steps.sum(1))))[0, 1]
        print("warp cost", col, ideal, learned, shuffled, "spearman", rho)
        assert ideal <= learned < 0.92 * shuffled, (col, ideal, learned, shuffled)
        assert rho > 0.3, rho


def test_training_is_deterministic():
    """Split-K sums its K-slices in a fixed order: two trainings from the same
    seed on the same batches give identical weights."""
    uv_h, seeds_h = _uv_grid(5, nx=64, ny=60)
    uv, seeds = torch.from_numpy(uv_h).to(DEV), torch.from_numpy(seeds_h).to(DEV)
    t = torch.rand((seeds.shape[0], 2), generator=torch.Generator().manual_seed(3)).to(DEV) * 5.0
    weights = []
    for _ in range(2):
        m = S.LengthModel(DEV, seed=0)
        m.fit(uv, uv.shape[0], uv.shape[1], 2, seeds, t, steps=60, batch=512)
        torch.cuda.synchronize()
        weights.append(m.master.clone())
    assert torch.equal(weights[0], weights[1])


def _time_ms(fn, reps=5):
    ts = []
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts[1:]))


def test_learned_order_timed_on_the_kernels():
    """The learned order on the real field kernels of a held-out 2048^2 DTM
    (the time includes inference and ordering).  With one thread per
    trajectory it is faster than the reference's shuffled order.  On the
    persistent pair launch, whose queue leaves little to order (even the
    true lengths gain 4.4 % over the spatial order at 2048^2), its
    predicted-long-first order stays within 25 % of the spatial order (both
    printed).  A 512^2 DTM is too small for this: there the plain kernel runs
    about three waves and its time is the longest warps' tail."""
    m, hist, *_ = _trained_and_eval()
    ev = Workload("incised2048")
    seeds = torch.from_numpy(ev.seeds).to(DEV)
    mask = torch.from_numpy(ev.mask.view(np.uint8)).to(DEV)
    uv = torch.from_numpy(ev.uv).to(DEV)
    prm = kernel_params(ev.info, "INTEGRATE_FIELDS", 1.0)
    n = int(ev.info.n_seed_points)
    nxy = int(prm.nxy_padded)
    p = [kernel_params(ev.info, "INTEGRATE_FIELDS", sg) for sg in (1.0, -1.0)]
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=DEV)
    work = kernels.workspace(DEV)
    cap = S.log_cap(prm)
    thr = [float(torch.quantile(m.predict(uv, uv.shape[0], uv.shape[1], 2, seeds, n)[:, c], 0.99)) for c in (0, 1)]

    def plain(order_fn):
        acc.zero_()
        orders = order_fn()
        for c in (0, 1):
            kernels.integrate_fields(p[c], seeds, mask, uv, acc[c, 0], acc[c, 1], work, schedule="plain",
                                     integrator=ev.spec.integrator, order=orders[c])

    def learned():
        pred = m.predict(uv, uv.shape[0], uv.shape[1], 2, seeds, n)
        return [m.order(pred, c, cap) for c in (0, 1)]

    def pair(order_fn):
        acc.zero_()
        o = order_fn()
        kernels.integrate_fields_pair(p[0], p[1], seeds, mask, uv, acc[:, 0], acc[:, 1], work,
                                      integrator=ev.spec.integrator, order=o[0], order_up=o[1])

    def spatial():
        o = S.spatial_order(seeds, n, ev.info.nx, ev.info.ny)
        return [o, o]

    def learned_spatial():
        pred = m.predict(uv, uv.shape[0], uv.shape[1], 2, seeds, n)
        return [S.spatial_order(seeds, n, ev.info.nx, ev.info.ny, pred=pred, col=c, threshold=thr[c])
                for c in (0, 1)]

    results = {}
    ref = None
    for name, fn in (("plain_shuffled", lambda: plain(lambda: [None, None])), ("plain_learned", lambda: plain(learned)),
                     ("pair_spatial", lambda: pair(spatial)), ("pair_learned_spatial", lambda: pair(learned_spatial))):
        fn()
        torch.cuda.synchronize()
        if ref is None:
            ref = acc.clone()
        assert torch.equal(acc, ref), name
        results[name] = _time_ms(fn)
    print("learned order, ms:", results)
    assert results["plain_learned"] < results["plain_shuffled"], results
    assert results["pair_learned_spatial"] < 1.25 * results["pair_spatial"], results


@pytest.mark.parametrize("block", [64, 4])  # 64: bins counted in shared memory; 4: 5625 bins, global
@pytest.mark.parametrize("with_pred", [False, True])
def test_spatial_order(block, with_pred):
    rng = np.random.default_rng(10)
    nx, ny, n = 300, 300, 70001
    seeds = np.stack([rng.integers(0, nx, n), rng.integers(0, ny, n)], 1).astype(np.float32)
    seeds[3] = [np.nan, -5.0]  # clamped into the grid
    pred = rng.uniform(0, 8, (n, 2)).astype(np.float32)
    sd, pd = torch.from_numpy(seeds).to(DEV), torch.from_numpy(pred).to(DEV)
    order = S.spatial_order(sd, n, nx, ny, block=block, pred=pd if with_pred else None, col=1,
                            threshold=6.0).cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(n))
    xs = np.clip(np.nan_to_num(seeds[:, 0] + 0.5, nan=0.0), 0, nx - 1).astype(np.int64)
    ys = np.clip(np.nan_to_num(seeds[:, 1] + 0.5, nan=0.0), 0, ny - 1).astype(np.int64)
    nby = -(-ny // block)
    key = (xs // block) * nby + ys // block
    if with_pred:
        key = key + (pred[:, 1] < 6.0) * (-(-nx // block) * nby)
    assert np.all(np.diff(key[order]) >= 0)


def test_fields_spatial_order_identical():
    """Fields (the public API) traces in spatial order by default; the raw
    fields equal those of the reference's shuffled order."""
    from slm_b200.fields import Fields
    from slm_b200.useful import Data
    c = Case(nx=90, ny=70, seed=61, density=2, step=0.25, max_length=80.0)
    out = []
    for order in ("shuffled", "spatial"):
        data = Data(mask_array=c.mask, uv_array=c.uv)
        data.seed_point_array = c.seeds
        f = Fields(0, 0, info=c.info, data=data, seed_order=order)
        f.gpu_integrate()
        out.append((data.slc_array.copy(), data.slt_array.copy(), list(f.n_steps)))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2] == out[1][2] and out[0][2][0] > 0
