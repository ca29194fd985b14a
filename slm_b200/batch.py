"""Batched field tracing: many DTM tiles of uneven sizes traced in one
persistent work-queue launch per direction.

The reference traces one grid per ``Fields.integrate`` call, one
``integrate_fields`` kernel launch per direction (fields.py:69-310).  A
``TileBatch`` stores every tile's padded uv / mask grids and its seeds back to
back on the device, with a table of tiles (``slm_tile``: grid offset, padded
size, seed range and the grid-derived GRID_SCALE / COMBO_FACTOR / DT_MAX) per
direction; ``trace`` runs both directions over all tiles, each as a single
``slm_integrate_fields_batched`` launch.  Each tile's slc/slt equal what a
per-tile launch produces (``trace_per_tile``, the plain form kept for
comparison): the trajectories are the same, RNG stream of the tile-local seed
index included.  ``capture`` records zeroing + both directions in a CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, kernels, synth
from ._lib import SlmTile, check, ptr, sref
from .params import kernel_params
from .useful import Info, create_seeds, default_parameters

# parameters every tile of a batch must share (the kernel reads them once)
SHARED = ("integrator_step_factor", "max_integration_step_error", "adjusted_max_error",
          "integration_halt_threshold", "max_length", "pixel_size", "pad_width", "pad_width_pp5",
          "max_n_steps", "trajectory_resolution", "subpixel_seed_point_density",
          "subpixel_seed_halfspan", "subpixel_seed_step", "jitter_magnitude", "downup_sign")


class Tile:
    """One DTM tile: padded uv / mask, Info and its shuffled seed list."""

    def __init__(self, uv, mask, info, seeds):
        self.uv, self.mask, self.info, self.seeds = uv, mask, info, seeds

    @property
    def n_seeds(self):
        return int(self.info.n_seed_points)


def make_tile(dtm, pixel_size=1.0, density=2, jitter=1.0, step=0.1, max_steps=2000, pad=2,
              defaults=None):
    """Tile from a DTM the way Fields sees it: uv/mask (preprocess), Info, shuffled seeds."""
    d = defaults or default_parameters()
    d.trace.subpixel_seed_point_density = density
    d.trace.jitter_magnitude = jitter
    d.trace.integrator_step_factor = step
    d.trace.max_length = max_steps * step
    uv, mask = synth.uv_from_dtm(dtm, pixel_size, pad)
    info = Info(d.state, d.trace, pixel_size)
    info.set_xy(dtm.shape[0], dtm.shape[1], pad)
    seeds, ns, npad = create_seeds(mask, pad, info.n_work_items, do_shuffle=True, rng_seed=1)
    info.n_seed_points = ns
    info.n_padded_seed_points = npad
    return Tile(uv, mask, info, seeds)


def tile_table(tiles, sign):
    """(SlmTile array, shared SlmParams) of one direction; checks the batch."""
    prms = [kernel_params(t.info, "INTEGRATE_FIELDS", sign) for t in tiles]
    table = (SlmTile * len(tiles))()
    off = seed = 0
    for i, (t, p) in enumerate(zip(tiles, prms)):
        for name in SHARED:
            if getattr(p, name) != getattr(prms[0], name):
                raise ValueError("tile {} differs from tile 0 in {}".format(i, name))
        if t.n_seeds and t.seeds.shape[0] < t.n_seeds:
            raise ValueError("tile {} has fewer seeds than n_seed_points".format(i))
        e = table[i]
        e.grid_offset = off
        e.nx_padded, e.ny_padded = p.nx_padded, p.ny_padded
        e.seed_begin, e.n_seeds = seed, t.n_seeds
        e.grid_scale, e.combo_factor, e.dt_max = p.grid_scale, p.combo_factor, p.dt_max
        off += int(p.nxy_padded)
        seed += t.n_seeds
    if off >= 2 ** 32:
        raise ValueError("a batch holds fewer than 2^32 padded pixels")
    shared = prms[0]
    shared.n_seed_points = seed
    shared.seeds_chunk_offset = 0
    return table, shared, off, seed


class TileBatch:
    """Device-resident batch of tiles with accumulators for both directions."""

    def __init__(self, tiles, device=None, integrator=2, seed_order="spatial"):
        self.tiles = list(tiles)
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self.integrator = int(integrator)
        self.tables, self.shared = [], []
        for sign in (1.0, -1.0):
            table, shared, n_px, n_seeds = tile_table(self.tiles, sign)
            raw = np.frombuffer(bytes(table), dtype=np.uint8).copy()
            self.tables.append(torch.from_numpy(raw).to(self.device))
            self.shared.append(shared)
        self.n_px, self.n_seeds = n_px, n_seeds
        self.grid_offsets = [int(table[i].grid_offset) for i in range(len(self.tiles))]
        self.seed_begins = [int(table[i].seed_begin) for i in range(len(self.tiles))]
        dev = self.device
        self.uv = torch.from_numpy(np.concatenate(
            [t.uv.reshape(-1, 2) for t in self.tiles]).astype(np.float32)).to(dev)
        self.mask = torch.from_numpy(np.concatenate(
            [t.mask.reshape(-1).view(np.uint8) for t in self.tiles])).to(dev)
        seeds = [t.seeds[:t.n_seeds] for t in self.tiles]
        self.seeds = torch.from_numpy(np.ascontiguousarray(
            np.concatenate(seeds) if self.n_seeds else np.zeros((1, 2), np.float32))).to(dev)
        self.acc = torch.zeros((2, 2, max(1, self.n_px)), dtype=torch.uint64, device=dev)
        self.work = [kernels.workspace(dev) for _ in range(2)]
        self.launch = kernels.launch_config("persistent", self.integrator)
        self._graph = None
        # queue order: each tile's seeds in pixel-block order (the tiles in
        # table order), as global seed indices; None = the seed arrays' order
        self.order = None
        if seed_order == "spatial" and self.n_seeds:
            from .scheduler import spatial_order
            parts = []
            for t, b in zip(self.tiles, self.seed_begins):
                if t.n_seeds:
                    o = spatial_order(self.seeds[b:b + t.n_seeds], t.n_seeds, t.info.nx, t.info.ny)
                    parts.append(o.view(torch.int32) + b)
            self.order = torch.cat(parts).contiguous().view(torch.uint32)
        elif seed_order not in ("spatial", "shuffled"):
            raise ValueError("seed_order must be 'spatial' or 'shuffled'")

    # ------------------------------------------------------------ tracing
    def trace_direction(self, d, launch=None, order=None, item_steps=None, stream=None):
        """One direction over all tiles; ``order`` defaults to the batch's queue order."""
        order = self.order if order is None else order
        L = launch if launch is not None else self.launch
        L.integrator = self.integrator
        lib = _lib.load()
        check(lib.slm_integrate_fields_batched(
            sref(self.shared[d]), sref(L), ptr(self.tables[d]), len(self.tiles), self.n_seeds,
            ptr(self.seeds), ptr(self.mask), ptr(self.uv), ptr(self.acc[d, 0]), ptr(self.acc[d, 1]),
            ptr(self.work[d]), ptr(order), ptr(item_steps), kernels._stream(stream)))

    def trace(self, launch=None, stream=None):
        """Zero the accumulators and trace both directions (2 batched launches)."""
        self.acc.zero_()
        for d in range(2):
            self.trace_direction(d, launch, stream=stream)

    def trace_per_tile(self, schedule="persistent", block_threads=0, stream=None):
        """The plain form: one field launch per tile and direction."""
        self.acc.zero_()
        if not hasattr(self, "work_tiles"):
            self.work_tiles = [[kernels.workspace(self.device) for _ in self.tiles] for _ in range(2)]
            self.tile_prm = [[kernel_params(t.info, "INTEGRATE_FIELDS", sign) for t in self.tiles]
                             for sign in (1.0, -1.0)]
            # each tile's own slice of the queue order, as tile-local indices
            self._tile_orders = []
            for t, b in zip(self.tiles, self.seed_begins):
                if self.order is None or t.n_seeds == 0:
                    self._tile_orders.append(None)
                else:
                    sl = self.order.view(torch.int32)[b:b + t.n_seeds] - b
                    self._tile_orders.append(sl.contiguous().view(torch.uint32))
        for d in range(2):
            for i, t in enumerate(self.tiles):
                self.work_tiles[d][i].zero_()
                if t.n_seeds == 0:
                    continue
                prm = self.tile_prm[d][i]
                o, n = self.grid_offsets[i], int(prm.nxy_padded)
                b = self.seed_begins[i]
                kernels.integrate_fields(prm, self.seeds[b:b + t.n_seeds], self.mask[o:o + n],
                                         self.uv[o:o + n], self.acc[d, 0, o:o + n],
                                         self.acc[d, 1, o:o + n], self.work_tiles[d][i], schedule=schedule,
                                         integrator=self.integrator, block_threads=block_threads,
                                         stream=stream, order=self._tile_orders[i])

    def capture(self, launch=None):
        """CUDA graph of zeroing + both batched directions; returns it (also kept)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.trace(launch, stream=s)  # warm-up outside capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.trace(launch, stream=torch.cuda.current_stream(self.device))
        self._graph = g
        return g

    # ------------------------------------------------------------ results
    def field_steps(self, per_tile=False):
        """RK steps of the last trace (batched, or per-tile with per_tile=True)."""
        if per_tile:
            return sum(int(w[1].item()) for ws in self.work_tiles for w in ws)
        return sum(int(w[1].item()) for w in self.work)

    def status(self):
        return max(int(w[3].item()) for w in self.work)

    def tile_fields(self, i):
        """(slc, slt) uint64 [2, nxp, nyp] of tile i (device views)."""
        t = self.tiles[i]
        o, n = self.grid_offsets[i], int(t.info.nx_padded) * int(t.info.ny_padded)
        shape = (2, int(t.info.nx_padded), int(t.info.ny_padded))
        return self.acc[:, 0, o:o + n].reshape(shape), self.acc[:, 1, o:o + n].reshape(shape)


def shard_tiles(sizes, rank, world_size):
    """Indices of the tiles rank ``rank`` of ``world_size`` traces: whole tiles,
    largest first onto the least-loaded rank (ties to the lower rank), so the
    ranks' pixel counts balance and every tile is traced exactly once.  Tiles
    are independent (own grids, own fields), so sharding needs no collective
    beyond gathering the ranks' counters."""
    if not 0 <= rank < world_size:
        raise ValueError("rank {} outside world size {}".format(rank, world_size))
    load = [0] * world_size
    mine = []
    for i in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world_size), key=lambda k: (load[k], k))
        load[r] += int(sizes[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)


def uneven_tiles(n_tiles=96, lo=256, hi=3072, seed=3, **kw):
    """``n_tiles`` fBm tiles (tilt + hills + fBm, each its own seed, hills cut
    at 5 sigma) with edge lengths log-uniform in [lo, hi] px, each edge drawn
    independently."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_tiles):
        nx, ny = (int(round(np.exp(rng.uniform(np.log(lo), np.log(hi))))) for _ in range(2))
        out.append(make_tile(synth.tile_dtm(nx, ny, 1000 + seed * 1000 + i, hill_truncate=5.0), **kw))
    return out
