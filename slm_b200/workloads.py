"""Named synthetic workloads (DTM recipe + trace parameters) for the bench and tests.

Each workload is one of the configurations the tracer is measured on; the
DTMs are seeded synthetic stand-ins (slm_b200.synth) for lidar DTMs.
"step" is ``integrator_step_factor`` (the maximum step in px) and the step cap
is set the way the reference derives it, ``max_n_steps = max_length / step``
(useful.py:159), with ``max_length = cap * step`` in metres.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import synth
from .useful import Info, create_seeds, default_parameters


@dataclass
class WorkloadSpec:
    name: str
    n: int
    pixel_size: float
    density: int
    jitter: float
    integrator: int
    step: float
    max_steps: int
    dtm: str
    n_traj_seeds: int = 1000
    cpu_stride: int = 0  # seed stride of the host-core sample (0: sized to the time budget)


SPECS = {
    "hills512": WorkloadSpec("512x512 @1m, d=1, no jitter, RK2, step 0.1 px, max 2000 steps",
                            512, 1.0, 1, 0.0, 2, 0.1, 2000, "hills"),
    "incised2048": WorkloadSpec("2048x2048 @2m, d=2, jitter +-0.5, RK4, step 0.1 px, max 10000 steps",
                            2048, 2.0, 2, 1.0, 4, 0.1, 10000, "incised"),
    "incised2048_rk2": WorkloadSpec("2048x2048 @2m, d=2, jitter +-0.5, RK2, step 0.1 px, max 10000 steps",
                                2048, 2.0, 2, 1.0, 2, 0.1, 10000, "incised"),
    "fan8192": WorkloadSpec("8192x8192 @1m, d=2, jitter +-0.5, RK4, step 0.1 px, max 20000 steps",
                            8192, 1.0, 2, 1.0, 4, 0.1, 20000, "fan", cpu_stride=64),
    "fan8192_rk2": WorkloadSpec("8192x8192 @1m, d=2, jitter +-0.5, RK2, step 0.1 px, max 20000 steps",
                                8192, 1.0, 2, 1.0, 2, 0.1, 20000, "fan", cpu_stride=256),
    # the fan family at a quarter of the area, one seed per pixel: a case
    # whose uv (134 MB) exceeds L2 and which fits a profiler capture
    "fan4096_d1": WorkloadSpec("4096x4096 @1m fan, d=1, jitter +-0.5, RK4, step 0.1 px, max 20000 steps",
                               4096, 1.0, 1, 1.0, 4, 0.1, 20000, "fan"),
    "tile256": WorkloadSpec("256x256 @1m, d=2, jitter +-0.5, RK2, step 0.1 px, max 2000 steps",
                          256, 1.0, 2, 1.0, 2, 0.1, 2000, "tile"),
    "incised4096_d4": WorkloadSpec("4096x4096 @2m incised fBm, d=4, jitter +-0.5, RK4, step 0.1 px, "
                            "max 10000 steps", 4096, 2.0, 4, 1.0, 4, 0.1, 10000, "incised"),
    "incised512_d4": WorkloadSpec("512x512 @2m incised fBm, d=4, jitter +-0.5, RK4, step 0.1 px, "
                                  "max 10000 steps", 512, 2.0, 4, 1.0, 4, 0.1, 10000, "incised"),
    "incised512": WorkloadSpec("512x512 @2m incised fBm, d=2, jitter +-0.5, RK2, step 0.1 px, "
                               "max 10000 steps", 512, 2.0, 2, 1.0, 2, 0.1, 10000, "incised"),
}


def make_dtm(spec, seed=None):
    if spec.dtm == "hills":
        return synth.hills_dtm(spec.n, seed or 1)
    if spec.dtm == "fan":  # 5000 pits per 8192^2, scaled by area
        return synth.fan_dtm(spec.n, seed or 5, max(8, round(5000 * spec.n * spec.n / 8192 ** 2)))
    if spec.dtm == "incised":  # 400 incisions per 2048^2, scaled by area
        return synth.incised_dtm(spec.n, seed or 2, max(8, round(400 * spec.n * spec.n / 2048 ** 2)))
    return synth.tile_dtm(spec.n, spec.n, seed or 9)


def numpy_seeds(mask, pad, rng_seed=1):
    """The field seed list built the reference's way, in NumPy alone
    (useful.py:496-501): argwhere of the unmasked pixels minus the pad,
    shuffled by NumPy's global legacy generator seeded with ``rng_seed``."""
    seeds = np.argwhere(~mask).astype(np.float32) - pad
    np.random.seed(rng_seed)
    np.random.shuffle(seeds)
    return seeds


class Workload:
    """DTM, uv, mask, Info and the shuffled seed lists of one configuration.

    ``seed_list="native"`` shuffles with the library's host code
    (``slm_create_seeds``); ``"numpy"`` with NumPy's own shuffle, for callers
    that must not load the library (the same list)."""

    def __init__(self, key, seed=None, seed_list="native"):
        spec = SPECS[key]
        self.key = key
        self.spec = spec
        self.dtm = make_dtm(spec, seed)
        self.uv, self.mask = synth.uv_from_dtm(self.dtm, spec.pixel_size, 2)
        d = default_parameters()
        d.trace.subpixel_seed_point_density = spec.density
        d.trace.jitter_magnitude = spec.jitter
        d.trace.integrator_step_factor = spec.step
        d.trace.max_length = spec.max_steps * spec.step
        d.trace.n_trajectory_seed_points = spec.n_traj_seeds
        self.defaults = d
        self.info = Info(d.state, d.trace, spec.pixel_size)
        self.info.set_xy(spec.n, spec.n, 2)
        if seed_list == "numpy":
            self.seeds = numpy_seeds(self.mask, 2, 1)
            ns = self.seeds.shape[0]
            wi = int(self.info.n_work_items)
            npad = ns + (int(np.round(ns / wi + 0.5)) * wi - ns)
        else:
            self.seeds, ns, npad = create_seeds(self.mask, 2, self.info.n_work_items,
                                                do_shuffle=True, rng_seed=1)
        self.info.n_seed_points = ns
        self.info.n_padded_seed_points = npad
        self.traj_seeds = np.ascontiguousarray(self.seeds[:spec.n_traj_seeds])
        self.n_traj = min(spec.n_traj_seeds, ns)

    @property
    def n_pixels(self):
        return self.spec.n * self.spec.n

    def fresh_info(self):
        i = Info(self.defaults.state, self.defaults.trace, self.spec.pixel_size)
        i.set_xy(self.spec.n, self.spec.n, 2)
        return i
