"""The oracle's C restatement against the reference's own kernel at the
2048^2 workload's full DTM size (CPU).

Every 64th seed of the incised 2048^2 DTM's shuffled list (65 K seeds, d=2,
jitter +-0.5 px, RK2, step 0.1 px, max 10000 steps), both directions: the
restatement's uint64 slc/slt, reduced mod 2^32, equal the uint32 arrays of
the reference's integrate_fields (opencl/integratefields.cl:60-114) compiled
for the host.  This pins the restatement on the same inputs the GPU parity
test at this size compares against.
"""
import os

import numpy as np
import pytest

import oracle as O
from slm_b200.params import kernel_params
from slm_b200.workloads import Workload


def test_restatement_equals_reference_kernel_at_2048():
    if not O.ref_available("integrate_fields"):
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")
    wl = Workload("incised2048_rk2")
    sub = np.ascontiguousarray(wl.seeds[::64])
    cores = os.cpu_count() or 1
    for sign in (1.0, -1.0):
        prm = kernel_params(wl.info, "INTEGRATE_FIELDS", sign)
        prm.n_seed_points = sub.shape[0]
        slc, slt, steps, _ = O.integrate_fields(prm, sub, wl.mask, wl.uv, 2, n_threads=cores)
        rslc, rslt = O.ref_integrate_fields(prm, sub, wl.mask, wl.uv, n_threads=cores)
        assert steps > 10_000_000
        assert np.array_equal((slc & np.uint64(0xFFFFFFFF)).astype(np.uint32), rslc)
        assert np.array_equal((slt & np.uint64(0xFFFFFFFF)).astype(np.uint32), rslt)
