"""Multi-rank seed sharding and the uint64 all-reduce, on CPU ranks (gloo).

Each rank traces its dealt share of the queue with the oracle standing in for
the device kernel (the dealing and reduction logic is the product's); the
reduced slc/slt must equal a single-rank trace bit for bit, at world sizes 2
and 3.  The dealing's load balance is measured on per-seed step counts the
oracle records on an incised DTM.
"""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from cases import Case
from slm_b200 import distributed as D


def _case():
    return Case(nx=40, ny=36, seed=71, density=2, jitter=1.0, step=0.25, max_length=60.0)


def _runs(queue):
    """Split ascending seed indices into contiguous [begin, end) runs."""
    q = np.asarray(queue, np.int64)
    if q.size == 0:
        return []
    cut = np.flatnonzero(np.diff(q) != 1) + 1
    return [(int(r[0]), int(r[-1]) + 1) for r in np.split(q, cut)]


def _oracle_trace(c):
    """The oracle standing in for the device trace of a queue of seed indices
    (the queue of the seed list's own order: ascending runs)."""
    import oracle as O

    def fn(p, slc, slt, queue):
        a, b = slc.numpy(), slt.numpy()
        q = queue.view(torch.int32).numpy()
        full = c.params("INTEGRATE_FIELDS", 1.0).n_seed_points
        steps = 0
        for begin, end in _runs(q):
            prm = p.copy()
            prm.n_seed_points = full
            s, = (O.integrate_fields(prm, c.seeds, c.mask, c.uv, seed_begin=begin, seed_end=end,
                                     slc=a, slt=b)[2],)
            steps += s
        return steps
    return fn


def _worker(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle"), os.path.join(root, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        c = _case()
        prm = c.params("INTEGRATE_FIELDS", -1.0)
        nxy = prm.nxy_padded
        slc = torch.zeros(nxy, dtype=torch.uint64)
        slt = torch.zeros(nxy, dtype=torch.uint64)
        mine, total = D.sharded_field_pass(prm, _oracle_trace(c), slc, slt)
        np.save(os.path.join(out_dir, "slc_{}.npy".format(rank)), slc.numpy())
        np.save(os.path.join(out_dir, "slt_{}.npy".format(rank)), slt.numpy())
        np.save(os.path.join(out_dir, "steps_{}.npy".format(rank)), np.array([mine, total]))
    finally:
        dist.destroy_process_group()


def test_shard_ranges_cover_exactly():
    for n in (0, 1, 7, 1000, 4194304):
        for w in (1, 2, 3, 8):
            r = [D.shard_range(n, k, w) for k in range(w)]
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(r[k][1] == r[k + 1][0] for k in range(w - 1))


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 1000, 100003])
@pytest.mark.parametrize("w", [1, 2, 3, 8])
def test_dealt_queues_partition_the_queue(n, w):
    """Every queue position goes to exactly one rank; the device-side dealing
    (shard_queue) equals the host-side positions; queues follow the order."""
    pos = [D.shard_positions(n, r, w) for r in range(w)]
    allp = np.sort(np.concatenate(pos)) if pos else np.zeros(0)
    assert np.array_equal(allp, np.arange(n))
    order = torch.from_numpy(np.random.default_rng(n).permutation(n).astype(np.int32)).view(torch.uint32)
    for r in range(w):
        assert np.all(np.diff(pos[r]) > 0)
        q = D.shard_queue(order, n, r, w)
        assert np.array_equal(q.view(torch.int32).numpy(), order.view(torch.int32).numpy()[pos[r]])
        qi = D.shard_queue(None, n, r, w, device="cpu")
        assert np.array_equal(qi.view(torch.int32).numpy(), pos[r])
        assert D.shard_queue_params(_case().params("INTEGRATE_FIELDS", 1.0), q).n_seed_points == len(pos[r])


def _spatial_queue(seeds, nx, ny, block=64):
    """Seed indices by block x block pixel block, blocks x-major (the blocks
    of the tracer's spatial order; stable inside a block)."""
    bx = np.clip(np.floor(seeds[:, 0]).astype(np.int64), 0, nx - 1) // block
    by = np.clip(np.floor(seeds[:, 1]).astype(np.int64), 0, ny - 1) // block
    nby = (ny + block - 1) // block
    return np.argsort(bx * nby + by, kind="stable")


def test_dealt_shards_balance_the_load():
    """Per-rank load (the sum of the RK steps of its seeds) for contiguous
    ranges of the spatial queue and for the dealt chunks, at 2..8 ranks, on
    the per-seed step counts the oracle records on a 512^2 incised DTM
    (d=2, jitter +-0.5 px, RK2, step 0.1 px, max 10000 steps): the dealt
    chunks stay within 5 % of the mean at 8 ranks and beat the contiguous
    ranges' imbalance."""
    import oracle as O
    from slm_b200.params import kernel_params
    from slm_b200.workloads import Workload
    wl = Workload("incised512")
    prm = kernel_params(wl.info, "INTEGRATE_FIELDS", 1.0)
    steps = O.field_seed_steps(prm, wl.seeds, wl.mask, wl.uv, 2, n_threads=os.cpu_count() or 1).astype(np.int64)
    n = steps.size
    queue = _spatial_queue(wl.seeds, int(wl.info.nx), int(wl.info.ny))
    load_q = steps[queue]
    report = {}
    for w in range(2, 9):
        contiguous = [load_q[slice(*D.shard_range(n, r, w))].sum() for r in range(w)]
        dealt = [load_q[D.shard_positions(n, r, w)].sum() for r in range(w)]
        report[w] = (max(contiguous) / np.mean(contiguous), max(dealt) / np.mean(dealt))
    for w, (c_ratio, d_ratio) in report.items():
        assert d_ratio <= c_ratio + 1e-9, report
    assert report[8][1] <= 1.05, report
    assert report[8][0] > report[8][1], report


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_fields_equal_single_rank(world, tmp_path):
    import oracle as O
    c = _case()
    prm = c.params("INTEGRATE_FIELDS", -1.0)
    ref_slc, ref_slt, ref_steps, _ = O.integrate_fields(prm, c.seeds, c.mask, c.uv)
    port = 29500 + (os.getpid() % 1000) + world
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / "slc_{}.npy".format(r)), ref_slc)
        assert np.array_equal(np.load(tmp_path / "slt_{}.npy".format(r)), ref_slt)
        mine, total = np.load(tmp_path / "steps_{}.npy".format(r))
        assert total == ref_steps


def _failing_worker(rank, world, port, out_dir):
    """Rank 1's trace raises before the all-reduce; rank 0 records what its
    all-reduce does (it must fail within the group's short timeout, not hang)."""
    import sys
    import time
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle"), os.path.join(root, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    c = _case()
    prm = c.params("INTEGRATE_FIELDS", 1.0)
    nxy = prm.nxy_padded
    slc = torch.zeros(nxy, dtype=torch.uint64)
    slt = torch.zeros(nxy, dtype=torch.uint64)

    def trace(p, a, b, queue):
        if rank == 1:
            raise RuntimeError("injected failure on rank 1")
        return _oracle_trace(c)(p, a, b, queue)
    t0 = time.time()
    try:
        D.sharded_field_pass(prm, trace, slc, slt)
        outcome = "completed"
    except Exception as e:  # noqa: BLE001 - the outcome is what the test checks
        outcome = "{}: {}".format(type(e).__name__, str(e).splitlines()[0] if str(e) else "")
    with open(os.path.join(out_dir, "outcome_{}.txt".format(rank)), "w") as f:
        f.write("{}\n{:.1f}\n".format(outcome, time.time() - t0))
    if rank == 1:
        os._exit(3)  # the failed rank leaves without joining the collective
    try:
        dist.destroy_process_group()
    except Exception:  # noqa: BLE001
        pass


def test_failing_rank_ends_the_others_with_an_error(tmp_path):
    world = 2
    port = 29700 + (os.getpid() % 1000)
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_failing_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode is not None for p in procs), "a rank hung"
    assert procs[1].exitcode == 3
    r0 = (tmp_path / "outcome_0.txt").read_text().splitlines()
    r1 = (tmp_path / "outcome_1.txt").read_text().splitlines()
    assert r1[0].startswith("RuntimeError: injected failure")
    assert r0[0] != "completed" and float(r0[1]) < 60.0, r0
