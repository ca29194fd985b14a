"""GPU parity at the benchmarked configuration's full DTM size.

The 2048^2 incised DTM of the 2048^2 workload (fBm relief with 400 carved
valleys, d=2, jitter +-0.5 px, step 0.1 px, max 10000 steps) is traced on
the GPU over every 64th seed of its shuffled list (65 K seeds, 262 K
trajectories per direction that roam the whole grid), both directions in one
pair launch, and compared pixel for pixel over the full padded grid:

* RK2 against the reference's own integrate_fields kernel
  (opencl/integratefields.cl:60-114 with jittertrajectory.cl:42-88) compiled
  for the host; the reference keeps uint32 sums, so the GPU's low 32 bits;
* RK4 (this project's extension, no counterpart in the reference) against
  the oracle's C restatement, uint64 and the RK step count.

The sub-list is its own seed list (the RNG streams follow the position in
it), exactly what the host kernels trace.
"""
import os

import numpy as np
import pytest
import torch

import oracle as O
from slm_b200 import kernels
from slm_b200.params import kernel_params
from slm_b200.workloads import Workload

pytestmark = pytest.mark.gpu

DEV = "cuda"
STRIDE = 64


@pytest.fixture(scope="module")
def incised():
    return Workload("incised2048")


def _sub(wl):
    sub = np.ascontiguousarray(wl.seeds[::STRIDE])
    prm = [kernel_params(wl.info, "INTEGRATE_FIELDS", s) for s in (1.0, -1.0)]
    for p in prm:
        p.n_seed_points = sub.shape[0]
    return sub, prm


def _gpu_pair(wl, sub, prm, integrator):
    nxy = int(prm[0].nxy_padded)
    seeds = torch.from_numpy(sub).to(DEV)
    mask = torch.from_numpy(wl.mask.view(np.uint8)).to(DEV)
    uv = torch.from_numpy(wl.uv).to(DEV)
    acc = torch.zeros((2, 2, nxy), dtype=torch.uint64, device=DEV)
    work = kernels.workspace(DEV)
    kernels.integrate_fields_pair(prm[0], prm[1], seeds, mask, uv, acc[:, 0], acc[:, 1], work,
                                  integrator=integrator)
    torch.cuda.synchronize()
    return acc.cpu().numpy(), int(work[1].item())


def test_rk2_full_size_equals_reference_kernel(incised):
    if not O.ref_available("integrate_fields"):
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")
    sub, prm = _sub(incised)
    g, steps = _gpu_pair(incised, sub, prm, 2)
    assert steps > 10_000_000
    low = (g & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    for d in (0, 1):
        slc, slt = O.ref_integrate_fields(prm[d], sub, incised.mask, incised.uv, n_threads=os.cpu_count() or 1)
        assert slc.sum() > 0
        assert np.array_equal(low[d, 0], slc), "slc differs from the reference kernel (direction %d)" % d
        assert np.array_equal(low[d, 1], slt), "slt differs from the reference kernel (direction %d)" % d


def test_rk4_full_size_equals_restatement(incised):
    sub, prm = _sub(incised)
    g, steps = _gpu_pair(incised, sub, prm, 4)
    total = 0
    for d in (0, 1):
        slc, slt, n_steps, n_traj = O.integrate_fields(prm[d], sub, incised.mask, incised.uv, 4,
                                                       n_threads=os.cpu_count() or 1)
        assert n_traj == sub.shape[0] * 4
        assert np.array_equal(g[d, 0], slc), "slc differs from the restatement (direction %d)" % d
        assert np.array_equal(g[d, 1], slt), "slt differs from the restatement (direction %d)" % d
        total += n_steps
    assert steps == total
