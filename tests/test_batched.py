"""Host logic of batched tracing: tile tables, shared-parameter checks and the
slm_tile layout (CPU only)."""
import ctypes

import numpy as np
import pytest

from slm_b200 import batch, synth
from slm_b200._lib import SlmTile
from slm_b200.params import kernel_params


def _tiles():
    sizes = [(20, 33), (64, 40), (3, 3), (17, 51)]
    return [batch.make_tile(synth.tile_dtm(nx, ny, 50 + i), density=2, step=0.5, max_steps=100)
            for i, (nx, ny) in enumerate(sizes)]


def test_slm_tile_layout():
    assert ctypes.sizeof(SlmTile) == 40
    assert SlmTile.grid_offset.offset == 0 and SlmTile.seed_begin.offset == 16
    assert SlmTile.grid_scale.offset == 24 and SlmTile.dt_max.offset == 32


def test_tile_table_offsets_and_params():
    tiles = _tiles()
    for sign in (1.0, -1.0):
        table, shared, n_px, n_seeds = batch.tile_table(tiles, sign)
        off = seed = 0
        for i, t in enumerate(tiles):
            p = kernel_params(t.info, "INTEGRATE_FIELDS", sign)
            e = table[i]
            assert e.grid_offset == off and e.seed_begin == seed and e.n_seeds == t.n_seeds
            assert (e.nx_padded, e.ny_padded) == (p.nx_padded, p.ny_padded)
            assert np.float32(e.combo_factor) == np.float32(p.combo_factor)
            assert np.float32(e.grid_scale) == np.float32(p.grid_scale)
            assert np.float32(e.dt_max) == np.float32(p.dt_max)
            assert (e.combo_factor < 0) == (sign < 0)
            off += p.nxy_padded
            seed += t.n_seeds
        assert (n_px, n_seeds) == (off, seed) and shared.n_seed_points == seed


def test_tiles_must_share_trace_parameters():
    a = batch.make_tile(synth.tile_dtm(20, 20, 1), pixel_size=1.0, step=0.5, max_steps=100)
    b = batch.make_tile(synth.tile_dtm(20, 20, 2), pixel_size=2.0, step=0.5, max_steps=100)
    with pytest.raises(ValueError, match="differs"):
        batch.tile_table([a, b], 1.0)


def test_masked_tile_has_no_seeds():
    dtm = np.full((12, 9), np.nan, np.float32)
    t = batch.make_tile(dtm, step=0.5, max_steps=100)
    assert t.n_seeds == 0
    table, _, _, n_seeds = batch.tile_table(_tiles()[:1] + [t], 1.0)
    assert table[1].n_seeds == 0 and table[1].seed_begin == n_seeds


def test_uneven_tile_sizes():
    import slm_b200.batch as B
    rng = np.random.default_rng(3)
    edges = [int(round(np.exp(rng.uniform(np.log(256), np.log(3072))))) for _ in range(2 * 96)]
    assert 256 <= min(edges) and max(edges) <= 3072
    assert B.uneven_tiles.__defaults__[:3] == (96, 256, 3072)


def test_shard_tiles_whole_tiles_balanced():
    rng = np.random.default_rng(7)
    sizes = [int(np.exp(rng.uniform(np.log(256), np.log(3072)))) ** 2 for _ in range(96)]
    for ws in (1, 2, 3, 8):
        parts = [batch.shard_tiles(sizes, r, ws) for r in range(ws)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(96))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # LPT: every rank within the largest tile of the mean
        assert max(loads) - min(loads) <= max(sizes)
    with pytest.raises(ValueError):
        batch.shard_tiles(sizes, 2, 2)


def _gather_rank(rank, ws, port, sizes, q):
    import os
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    mine = batch.shard_tiles(sizes, rank, ws)
    t = torch.tensor([sum(sizes[i] for i in mine), len(mine)], dtype=torch.int64)
    dist.all_reduce(t)
    q.put((rank, int(t[0]), int(t[1])))
    dist.destroy_process_group()


def test_shard_tiles_gloo_gather():
    """Two gloo ranks shard the tiles and gather their counters: totals are
    the whole batch's (the only exchange the batched form needs)."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    sizes = [(50 + 7 * i) ** 2 for i in range(20)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(o[1] == sum(sizes) and o[2] == len(sizes) for o in out)
