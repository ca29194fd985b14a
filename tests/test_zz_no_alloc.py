"""slm_integrate_fields_noalloc against slm_integrate_fields, through the C ABI.

The no-alloc entry point serves callers that cannot call cudaMalloc (a host
application that only hands out its own pre-allocated device buffers, or a
binding of the reference's six-buffer kernel signature with no workspace
argument): it keeps the tracer's scratch in a static device array inside the
library.  Two calls in a row must each reproduce the workspace entry point's
slc/slt exactly (integer sums; the tolerance is zero), which also shows that
the shared scratch is cleared between calls.  This file is named so that
pytest collects it last.
"""
import ctypes

import numpy as np
import pytest
import torch

from cases import Case
from slm_b200 import _lib


def _call(fn_name, prm, launch, seeds, mask, uv, slc, slt, work=None):
    L = _lib.load()
    fn = getattr(L, fn_name)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = [_lib.sref(prm), _lib.sref(launch), _lib.ptr(seeds), _lib.ptr(mask), _lib.ptr(uv),
            None, _lib.ptr(slc), _lib.ptr(slt)]
    if work is not None:
        args.append(_lib.ptr(work))
    args.append(stream)
    _lib.check(fn(*args))


def test_noalloc_scratch_holds_the_tracer_workspace():
    """The static array must hold every scratch word the field tracer uses, so
    a tracer that grows its scratch fails here (CPU) before it could fail a
    caller (the entry point returns SLM_ERR_CAPACITY then)."""
    import os
    import re
    hdr = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "slm_b200.h")
    limit = int(re.search(r"#define SLM_NOALLOC_SCRATCH_WORDS (\d+)", open(hdr).read()).group(1))
    assert _lib.load().slm_fields_workspace_words() <= limit


@pytest.mark.gpu
@pytest.mark.parametrize("schedule,integrator", [(_lib.SLM_SCHED_PERSISTENT, _lib.SLM_RK2),
                                                 (_lib.SLM_SCHED_PLAIN, _lib.SLM_RK2),
                                                 (_lib.SLM_SCHED_PERSISTENT, _lib.SLM_RK4)])
def test_noalloc_matches_workspace_entry_point(schedule, integrator):
    c = Case(nx=72, ny=60, seed=61, density=2, jitter=1.0, step=0.25, max_length=90.0)
    dev = "cuda"
    seeds = torch.from_numpy(c.seeds).to(dev)
    mask = torch.from_numpy(c.mask.view(np.uint8)).to(dev)
    uv = torch.from_numpy(c.uv).to(dev)
    nxy = int(c.info.nx_padded * c.info.ny_padded)
    launch = _lib.SlmLaunch()
    launch.schedule = schedule
    launch.integrator = integrator
    work = torch.zeros(_lib.load().slm_fields_workspace_words(), dtype=torch.uint64, device=dev)
    for sign in (1.0, -1.0):
        prm = c.params("INTEGRATE_FIELDS", sign)
        ref_slc = torch.zeros(nxy, dtype=torch.uint64, device=dev)
        ref_slt = torch.zeros(nxy, dtype=torch.uint64, device=dev)
        _call("slm_integrate_fields", prm, launch, seeds, mask, uv, ref_slc, ref_slt, work)
        for _ in range(2):  # two calls in a row share the static scratch
            slc = torch.zeros(nxy, dtype=torch.uint64, device=dev)
            slt = torch.zeros(nxy, dtype=torch.uint64, device=dev)
            _call("slm_integrate_fields_noalloc", prm, launch, seeds, mask, uv, slc, slt)
            torch.cuda.synchronize()
            assert torch.equal(slc.view(torch.int64), ref_slc.view(torch.int64))
            assert torch.equal(slt.view(torch.int64), ref_slt.view(torch.int64))
