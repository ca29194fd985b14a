"""Seeded small test cases shared by the CPU and GPU tests."""
from __future__ import annotations

import numpy as np

from slm_b200 import params as P
from slm_b200 import synth
from slm_b200.useful import Info, create_seeds, default_parameters


class Case:
    """A synthetic DTM with its uv/mask, Info and shuffled seed list."""

    def __init__(self, nx=40, ny=56, seed=3, density=2, jitter=1.0, step=0.5, max_length=100.0,
                 pixel_size=1.0, n_traj_seeds=0, holes=False, pad=2):
        d = default_parameters()
        dtm = synth.tile_dtm(nx, ny, seed)
        if holes:
            rng = np.random.default_rng(seed + 100)
            for _ in range(3):
                cx, cy = rng.integers(4, nx - 4), rng.integers(4, ny - 4)
                dtm[cx - 2:cx + 2, cy - 1:cy + 3] = np.nan
        self.dtm = dtm
        self.uv, self.mask = synth.uv_from_dtm(dtm, pixel_size, pad)
        d.trace.subpixel_seed_point_density = density
        d.trace.jitter_magnitude = jitter
        d.trace.integrator_step_factor = step
        d.trace.max_length = max_length
        d.trace.n_trajectory_seed_points = n_traj_seeds
        self.defaults = d
        self.info = Info(d.state, d.trace, pixel_size)
        self.info.set_xy(nx, ny, pad)
        n = n_traj_seeds if n_traj_seeds > 0 else None
        self.seeds, ns, npad = create_seeds(self.mask, pad, self.info.n_work_items,
                                            n_seed_points=n, do_shuffle=True, rng_seed=1)
        self.info.n_seed_points = ns
        self.info.n_padded_seed_points = npad

    def params(self, kernel="INTEGRATE_FIELDS", sign=1.0):
        return P.kernel_params(self.info, kernel, sign)
