"""GPU parity of the batched multi-tile field tracer: each tile's slc/slt from
one batched launch equal the oracle's for that tile alone (bit-exact) and the
per-tile launches'; queue order and step recording change nothing; a CUDA
graph replays the same result; the autotuner picks and caches a shape."""
import numpy as np
import pytest
import torch

import oracle as O
from slm_b200 import autotune, batch, synth
from slm_b200.params import kernel_params

pytestmark = pytest.mark.gpu

DEV = "cuda"


def _tiles(integrator_seed=0):
    sizes = [(20, 33), (64, 40), (3, 3), (17, 51), (45, 45)]
    tiles = [batch.make_tile(synth.tile_dtm(nx, ny, 70 + i + integrator_seed), density=2, step=0.5,
                             max_steps=150) for i, (nx, ny) in enumerate(sizes)]
    dtm = np.full((12, 9), np.nan, np.float32)
    tiles.insert(2, batch.make_tile(dtm, density=2, step=0.5, max_steps=150))  # no seeds
    return tiles


def _oracle(tile, sign, integrator):
    prm = kernel_params(tile.info, "INTEGRATE_FIELDS", sign)
    if tile.n_seeds == 0:
        nxy = int(prm.nxy_padded)
        return np.zeros(nxy, np.uint64), np.zeros(nxy, np.uint64), 0
    slc, slt, steps, _ = O.integrate_fields(prm, tile.seeds, tile.mask, tile.uv,
                                            integrator=integrator, n_threads=4)
    return slc, slt, steps


@pytest.mark.parametrize("integrator", [2, 4])
def test_batched_matches_oracle_per_tile(integrator):
    tiles = _tiles(integrator)
    b = batch.TileBatch(tiles, DEV, integrator)
    b.trace()
    torch.cuda.synchronize()
    assert b.status() == 0
    total = 0
    for i, t in enumerate(tiles):
        slc, slt = b.tile_fields(i)
        for d, sign in enumerate((1.0, -1.0)):
            oslc, oslt, steps = _oracle(t, sign, integrator)
            assert np.array_equal(slc[d].cpu().numpy().ravel(), oslc), (i, d)
            assert np.array_equal(slt[d].cpu().numpy().ravel(), oslt), (i, d)
            total += steps
    assert b.field_steps() == total
    batched = b.acc.clone()
    for schedule in ("plain", "persistent"):
        b.trace_per_tile(schedule)
        torch.cuda.synchronize()
        assert torch.equal(b.acc, batched), schedule
        assert b.field_steps(per_tile=True) == total


def test_batched_order_and_steps():
    tiles = _tiles()
    b = batch.TileBatch(tiles, DEV, 2)
    b.trace()
    torch.cuda.synchronize()
    ref = b.acc.clone()
    dd = 4
    perm = torch.from_numpy(np.random.default_rng(1).permutation(b.n_seeds).astype(np.int32)).to(DEV)
    steps = [torch.zeros(b.n_seeds * dd, dtype=torch.uint16, device=DEV) for _ in range(2)]
    b.acc.zero_()
    for d in range(2):
        b.trace_direction(d, order=perm.view(torch.uint32), item_steps=steps[d])
    torch.cuda.synchronize()
    assert torch.equal(b.acc, ref)
    assert sum(int(s.to(torch.int64).sum()) for s in steps) == b.field_steps()


def test_graph_replay_identical():
    tiles = _tiles()
    b = batch.TileBatch(tiles, DEV, 4)
    b.trace()
    torch.cuda.synchronize()
    ref = b.acc.clone()
    g = b.capture()
    for _ in range(2):
        b.acc.fill_(7)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(b.acc, ref)


def test_autotune_picks_and_caches(tmp_path):
    tiles = _tiles()
    b = batch.TileBatch(tiles, DEV, 2)
    path = str(tmp_path / "tune.json")
    shapes = [(64, 8), (128, 4), (256, 2)]
    L, table = autotune.tune(lambda L: b.trace(L), "k_fields_batched", 2, "test", path=path,
                             shapes=shapes)
    assert set(table) == {"64x8", "128x4", "256x2"}
    assert (L.block_threads, L.blocks_per_sm) in shapes
    L2, table2 = autotune.tune(lambda L: b.trace(L), "k_fields_batched", 2, "test", path=path)
    assert table2 == {} and (L2.block_threads, L2.blocks_per_sm) == (L.block_threads, L.blocks_per_sm)
    ref = b.acc.clone()
    b.trace(L)
    torch.cuda.synchronize()
    assert torch.equal(b.acc, ref)
