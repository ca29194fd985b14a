"""Launch-shape autotuner for the persistent field kernels.

Times a caller-supplied run (one trace of a representative sample) for each
candidate launch shape -- threads per block x resident blocks per SM x refill
threshold (idle lanes a warp waits for before taking new work) -- with
CUDA events, keeps the fastest, and caches the choice in a JSON file keyed by
device name, kernel, integrator and a caller-given workload signature, so
later runs reuse it without tuning.
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np
import torch

from . import kernels

CACHE_PATH = os.environ.get(
    "SLM_AUTOTUNE_CACHE", os.path.join(os.path.dirname(os.path.abspath(__file__)), "_autotune.json"))
_lock = threading.Lock()

# (threads per block, resident blocks per SM, refill threshold): the
# threshold is slm_launch.chunk, the number of idle lanes a warp waits for
# before it takes new trajectories from the queue
CANDIDATES = [(256, 5, c) for c in (1, 2, 4, 8, 16)] + [(256, 4, c) for c in (1, 4)] \
    + [(128, 10, c) for c in (1, 4)] + [(128, 8, 4), (64, 20, 4), (64, 16, 4)]


def candidates():
    return list(CANDIDATES)


def _shape(c):
    return (c[0], c[1], c[2] if len(c) > 2 else 0)


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _key(kernel, integrator, signature):
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return "{}|{}|rk{}|{}".format(name, kernel, int(integrator), signature)


def tune(run, kernel, integrator, signature, reps=2, path=CACHE_PATH, force=False,
         shapes=None):
    """Best (block_threads, blocks_per_sm) for ``run(launch)``; cached.

    Returns ``(launch, table)`` where table maps "block x per_sm" to the
    median milliseconds (empty when the cache answered)."""
    key = _key(kernel, integrator, signature)
    with _lock:
        cache = _load(path)
    if not force and key in cache:
        e = cache[key]
        return kernels.launch_config("persistent", integrator, e["block_threads"], e["blocks_per_sm"],
                                     e.get("chunk", 1)), {}
    table = {}
    best = None
    for cand in (shapes or candidates()):
        b, k, c = _shape(cand)
        L = kernels.launch_config("persistent", integrator, b, k, c)
        run(L)  # warm-up
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            run(L)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        table["{}x{}" .format(b, k) + ("" if len(cand) == 2 else "/{}".format(c))] = ms
        if best is None or ms < best[0]:
            best = (ms, b, k, c)
    _, b, k, c = best
    with _lock:
        cache = _load(path)
        cache[key] = {"block_threads": b, "blocks_per_sm": k, "chunk": c, "ms": best[0], "table": table}
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return kernels.launch_config("persistent", integrator, b, k, c), table
