"""Launch-shape autotuner for the persistent field kernels.

Times a caller-supplied run (one trace of a representative sample) for each
candidate launch shape -- threads per block x resident blocks per SM -- with
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

# threads per block -> resident blocks per SM to try (bounded by the
# register-limited occupancy, which the library clamps to on launch)
CANDIDATES = {64: (8, 12, 16, 20), 128: (4, 6, 8, 10), 256: (2, 3, 4, 5)}


def candidates():
    return [(b, k) for b, ks in CANDIDATES.items() for k in ks]


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
        b, k = cache[key]["block_threads"], cache[key]["blocks_per_sm"]
        return kernels.launch_config("persistent", integrator, b, k), {}
    table = {}
    best = None
    for b, k in (shapes or candidates()):
        L = kernels.launch_config("persistent", integrator, b, k)
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
        table["{}x{}".format(b, k)] = ms
        if best is None or ms < best[0]:
            best = (ms, b, k)
    _, b, k = best
    with _lock:
        cache = _load(path)
        cache[key] = {"block_threads": b, "blocks_per_sm": k, "ms": best[0], "table": table}
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    return kernels.launch_config("persistent", integrator, b, k), table
