"""Multi-rank seed sharding and the uint64 all-reduce, on CPU ranks (gloo).

Each rank traces its seed shard with the oracle standing in for the device
kernel (the sharding and reduction logic is the product's); the reduced
slc/slt must equal a single-rank trace bit for bit, at world sizes 2 and 3.
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


def _oracle_trace(c):
    import oracle as O

    def fn(p, slc, slt):
        a, b = slc.numpy(), slt.numpy()
        _, _, steps, _ = O.integrate_fields(p, c.seeds, c.mask, c.uv, seed_begin=p.seeds_chunk_offset,
                                            seed_end=p.n_seed_points, slc=a, slt=b)
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

    def trace(p, a, b):
        if rank == 1:
            raise RuntimeError("injected failure on rank 1")
        return _oracle_trace(c)(p, a, b)
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
