"""GPU parity of the tracing kernels against the oracle (bit-exact).

Small cases are compared pixel for pixel with the oracle's C restatement
(itself pinned to the reference's kernels); larger ones through properties
that do not depend on size: schedule independence, visit/step accounting and
chunked-launch additivity.
"""
import numpy as np
import pytest
import torch

import oracle as O
from cases import Case
from slm_b200 import kernels

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _dev(c):
    seeds = torch.from_numpy(c.seeds).to(DEV)
    mask = torch.from_numpy(c.mask.view(np.uint8)).to(DEV)
    uv = torch.from_numpy(c.uv).to(DEV)
    return seeds, mask, uv


def _gpu_fields(c, prm, schedule, integrator=2, block=0):
    seeds, mask, uv = _dev(c)
    nxy = prm.nxy_padded
    slc = torch.zeros(nxy, dtype=torch.uint64, device=DEV)
    slt = torch.zeros(nxy, dtype=torch.uint64, device=DEV)
    work = kernels.workspace(DEV)
    kernels.integrate_fields(prm, seeds, mask, uv, slc, slt, work, schedule=schedule,
                             integrator=integrator, block_threads=block)
    torch.cuda.synchronize()
    w = work.cpu().numpy()
    return slc.cpu().numpy(), slt.cpu().numpy(), int(w[1]), int(w[2])


CASES = [
    dict(nx=40, ny=56, seed=3, density=2, jitter=1.0, step=0.5, max_length=100.0),
    dict(nx=33, ny=27, seed=5, density=3, jitter=0.5, step=0.1, max_length=30.0, holes=True),
    dict(nx=30, ny=30, seed=6, density=1, jitter=0.0, step=0.5, max_length=0.75),
    dict(nx=64, ny=48, seed=7, density=2, jitter=1.0, step=0.1, max_length=200.0, pixel_size=2.0),
]


@pytest.mark.parametrize("kw", CASES)
@pytest.mark.parametrize("schedule", ["plain", "persistent"])
@pytest.mark.parametrize("integrator", [2, 4])
def test_fields_bit_exact(kw, schedule, integrator):
    c = Case(**kw)
    for sign in (1.0, -1.0):
        prm = c.params("INTEGRATE_FIELDS", sign)
        oslc, oslt, osteps, ontraj = O.integrate_fields(prm, c.seeds, c.mask, c.uv,
                                                        integrator=integrator, n_threads=4)
        slc, slt, steps, ntraj = _gpu_fields(c, prm, schedule, integrator)
        assert np.array_equal(slc, oslc), "slc differs"
        assert np.array_equal(slt, oslt), "slt differs"
        assert steps == osteps and ntraj == ontraj


def test_fields_chunk_offset_additive():
    c = Case(nx=48, ny=40, seed=31, density=2)
    prm = c.params()
    full = _gpu_fields(c, prm, "persistent")
    c.info.seeds_chunk_offset = np.uint32(500)
    tail = _gpu_fields(c, c.params(), "persistent")
    c.info.seeds_chunk_offset = np.uint32(0)
    c.info.n_seed_points = np.uint32(500)
    head = _gpu_fields(c, c.params(), "plain")
    assert np.array_equal(head[0] + tail[0], full[0])
    assert np.array_equal(head[1] + tail[1], full[1])
    assert head[2] + tail[2] == full[2]


@pytest.mark.parametrize("block", [32, 96, 256])
def test_fields_launch_shapes_agree(block):
    c = Case(nx=80, ny=72, seed=41, density=2, step=0.25, max_length=120.0)
    prm = c.params("INTEGRATE_FIELDS", -1.0)
    a = _gpu_fields(c, prm, "plain", block=block)
    b = _gpu_fields(c, prm, "persistent", block=block)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_fields_large_properties():
    """256^2 grid, d=2: schedules agree; visits = steps + starts - masked exits."""
    c = Case(nx=256, ny=256, seed=51, density=2, step=0.1, max_length=200.0)
    prm = c.params()
    a = _gpu_fields(c, prm, "plain")
    b = _gpu_fields(c, prm, "persistent")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    visits, steps, ntraj = int(a[0].sum()), a[2], a[3]
    assert ntraj == int(prm.n_seed_points) * 4
    assert steps <= visits <= steps + ntraj
    # every unmasked seed pixel is visited at least by its own start
    assert np.all(a[0].reshape(c.mask.shape)[~c.mask] > 0)
    # oracle on a deterministic 1/97 stride of the seeds agrees with a GPU run on the same subset
    sub = np.ascontiguousarray(c.seeds[::97])
    c2 = Case(nx=256, ny=256, seed=51, density=2, step=0.1, max_length=200.0)
    c2.seeds = sub
    c2.info.n_seed_points = np.uint32(sub.shape[0])
    prm2 = c2.params()
    g = _gpu_fields(c2, prm2, "persistent")
    o = O.integrate_fields(prm2, sub, c.mask, c.uv, n_threads=4)
    assert np.array_equal(g[0], o[0]) and np.array_equal(g[1], o[1])


def _gpu_traj(c, prm, n, integrator=2):
    seeds, mask, uv = _dev(c)
    nl = prm.max_n_steps
    traj = torch.zeros(n * nl * 2, dtype=torch.int8, device=DEV)
    nsteps = torch.zeros(n, dtype=torch.uint16, device=DEV)
    length = torch.zeros(n, dtype=torch.float32, device=DEV)
    kernels.integrate_trajectory(prm, n, seeds, mask, uv, traj, nsteps, length, integrator)
    torch.cuda.synchronize()
    return traj.cpu().numpy().reshape(n, nl, 2), nsteps.cpu().numpy(), length.cpu().numpy()


@pytest.mark.parametrize("kw", [
    dict(nx=40, ny=40, seed=21, step=0.5, max_length=200.0, n_traj_seeds=200, holes=True),
    dict(nx=50, ny=30, seed=22, step=0.1, max_length=40.0, n_traj_seeds=100),
    dict(nx=96, ny=80, seed=24, step=0.1, max_length=200.0, n_traj_seeds=1000, holes=True),
])
@pytest.mark.parametrize("integrator", [2, 4])
def test_trajectory_bit_exact(kw, integrator):
    c = Case(**kw)
    n = int(c.info.n_seed_points)
    for sign in (np.float32(1.0), np.float32(-1.0)):
        prm = c.params("INTEGRATE_TRAJECTORY", sign)
        ot, on, ol, _ = O.integrate_trajectory(prm, n, c.seeds, c.mask, c.uv, integrator=integrator,
                                               n_threads=4)
        t, nn, ll = _gpu_traj(c, prm, n, integrator)
        assert np.array_equal(on, nn)
        assert np.array_equal(ol.view(np.uint32), ll.view(np.uint32))
        for k in range(n):
            assert np.array_equal(ot[k, :on[k]], t[k, :nn[k]]), k


def test_golden_on_gpu():
    """The GPU reproduces the reference's own golden outputs directly."""
    import glob
    import os
    from slm_b200 import params as P
    gdir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    for path in sorted(glob.glob(os.path.join(gdir, "fields_*.npz"))):
        g = np.load(path)
        c = Case(nx=4, ny=4)
        c.uv, c.mask, c.seeds = g["uv"], g["mask"], g["seeds"]
        for tag in ("down", "up"):
            prm = P.params_from_options(list(g["options_" + tag]))
            slc, slt, _, _ = _gpu_fields(c, prm, "persistent")
            assert np.array_equal(slc.astype(np.uint32), g["slc_" + tag])
            assert np.array_equal((slt & 0xFFFFFFFF).astype(np.uint32), g["slt_" + tag])


@pytest.mark.parametrize("integrator,ordered,interleaved", [(2, False, False), (4, False, False),
                                                            (2, True, False), (4, True, True),
                                                            (4, "per-direction", False)])
def test_fields_pair_equals_two_directions(integrator, ordered, interleaved):
    """One launch over both directions gives each direction's fields and the
    summed step and trajectory counts of two single-direction launches; the
    upstream rows may sit at any stride (interleaved: [direction][slc|slt]);
    the two directions may take their queues in different orders."""
    c = Case(nx=70, ny=58, seed=91, density=2, step=0.25, max_length=120.0)
    seeds, mask, uv = _dev(c)
    pd, pu = c.params("INTEGRATE_FIELDS", 1.0), c.params("INTEGRATE_FIELDS", -1.0)
    nxy = pd.nxy_padded
    order = order_up = None

    def perm(seed):
        p = np.random.default_rng(seed).permutation(int(pd.n_seed_points)).astype(np.int32)
        return torch.from_numpy(p).to(DEV).view(torch.uint32)

    if ordered:
        order = perm(5)
    if ordered == "per-direction":
        order_up = perm(6)
    ref = []
    for prm in (pd, pu):
        slc = torch.zeros(nxy, dtype=torch.uint64, device=DEV)
        slt = torch.zeros(nxy, dtype=torch.uint64, device=DEV)
        work = kernels.workspace(DEV)
        kernels.integrate_fields(prm, seeds, mask, uv, slc, slt, work, integrator=integrator)
        torch.cuda.synchronize()
        ref.append((slc.cpu().numpy(), slt.cpu().numpy(), int(work[1].item()), int(work[2].item())))
    if interleaved:
        acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=DEV)
        slc2, slt2 = acc[:, 0], acc[:, 1]
    else:
        slc2 = torch.zeros((2, nxy), dtype=torch.uint64, device=DEV)
        slt2 = torch.zeros((2, nxy), dtype=torch.uint64, device=DEV)
    work = kernels.workspace(DEV)
    kernels.integrate_fields_pair(pd, pu, seeds, mask, uv, slc2, slt2, work, integrator=integrator, order=order,
                                  order_up=order_up)
    torch.cuda.synchronize()
    for d in range(2):
        assert np.array_equal(slc2[d].cpu().numpy(), ref[d][0])
        assert np.array_equal(slt2[d].cpu().numpy(), ref[d][1])
    assert int(work[1].item()) == ref[0][2] + ref[1][2]
    assert int(work[2].item()) == ref[0][3] + ref[1][3]
    assert int(work[3].item()) == ref[1][2]


def test_division_free_sixth_is_exact_for_every_float():
    """The RK4 step's x / 6 is a product by 1/6 held as two floats (one fused
    multiply-add, no division) for finite |x| >= 2^-120, a division
    otherwise; over all 2^32 float bit patterns it equals the IEEE quotient
    x / 6.0f (NaN for NaN)."""
    import ctypes

    from slm_b200 import _lib
    counts = torch.zeros(2, dtype=torch.uint64, device=DEV)
    _lib.check(_lib.load().slm_selftest_div6(_lib.ptr(counts), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    bad, last = (int(v) for v in counts.view(torch.int64).cpu().tolist())
    assert bad == 0, "{} inputs differ, e.g. bit pattern {:#010x}".format(bad, last - 1)


def test_float_to_char_matches_x86_for_every_float():
    """The step quantisation's float -> char (one range test around the
    device's saturating conversion) equals the x86 conversion the reference
    follows over all 2^32 float bit patterns: truncation in range, low byte
    of INT32_MIN (0) for NaN and out of range."""
    import ctypes

    from slm_b200 import _lib
    counts = torch.zeros(2, dtype=torch.uint64, device=DEV)
    _lib.check(_lib.load().slm_selftest_cvt_i8(_lib.ptr(counts),
                                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    bad, last = (int(v) for v in counts.view(torch.int64).cpu().tolist())
    assert bad == 0, "{} inputs differ, e.g. bit pattern {:#010x}".format(bad, last - 1)
