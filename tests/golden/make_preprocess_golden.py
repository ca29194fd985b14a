#!/usr/bin/env python3
"""Generate the preprocess golden vectors from the reference's own Python.

Loads python/streamlines/preprocess.py from the reference checkout with two
stand-ins: numba's ``njit`` becomes the identity (the functions run as plain
Python/NumPy) and ``streamlines.core.Core`` an empty base class.  Then it
runs the reference's own ``Preprocess.find_blockages``,
``conditioned_gradient_vector_field`` and ``mask_nan_uv`` on seeded synthetic
ROIs and stores inputs and outputs as ``preprocess_*.npz``.

Two adjustments keep the plain-Python run on the numba build's semantics:

- ``np.hypot`` of the int8 flow-vector components (break_out_of_loop) runs
  on float32, the loop numba selects; plain NumPy would pick float16.
- ``np.dot(velocity, velocity)`` (check_has_loop) runs in double: numba
  types ``velocity / 4.0`` as a float64 array, plain NumPy as float32.
- the thresholds are passed as float64 scalars, so that the float32 speed,
  divergence and curl compare in double as in the numba build.

The loop detection visits cells 0..nx-2 x 0..ny-2: the reference's last row
and column of cells read one pixel beyond the grid (undefined in numba, an
IndexError in NumPy) and cannot change the field.

Usage: python tests/golden/make_preprocess_golden.py [reference checkout]
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $SLM_REFERENCE, else a "reference" folder beside the repository
DEFAULT_REF = os.environ.get("SLM_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")

CASES = {
    "preprocess_a": dict(nx=48, ny=40, seed=21, pixel_size=1.0, pad=2, noise=0.1),
    "preprocess_b": dict(nx=37, ny=52, seed=22, pixel_size=2.0, pad=3, noise=0.2, holes=True),
    "preprocess_c": dict(nx=41, ny=33, seed=23, pixel_size=0.7, pad=2, noise=0.1, normalize=False),
    "preprocess_d": dict(nx=30, ny=45, seed=24, pixel_size=1.5, pad=1, noise=0.1, dtype="float64",
                         plateaus=True),
    "preprocess_e": dict(nx=64, ny=64, seed=25, pixel_size=1.0, pad=2, noise=0.05, pits=True),
    # edge cases: the smallest grid, and a flat plateau (exact ties everywhere)
    # with one pit and a hole
    "preprocess_f": dict(nx=2, ny=2, seed=26, pixel_size=1.0, pad=1, noise=1.0),
    "preprocess_g": dict(nx=23, ny=19, seed=27, pixel_size=1.0, pad=2, noise=0.0, flat=True),
}
# The reference stores four pixels per looped cell in an nx*ny array, so at
# most a quarter of the cells may loop; the noise levels stay well below.


def load_reference_preprocess(ref=DEFAULT_REF):
    numba = types.ModuleType("numba")
    dec = types.ModuleType("numba.decorators")

    def njit(*a, **k):
        if a and callable(a[0]):
            return a[0]
        return lambda f: f
    dec.njit = njit
    numba.decorators = dec
    core = types.ModuleType("streamlines.core")
    core.Core = type("Core", (), {})
    pkg = types.ModuleType("streamlines")
    pkg.core = core
    saved = {k: sys.modules.get(k) for k in ("numba", "numba.decorators", "streamlines", "streamlines.core")}
    sys.modules.update({"numba": numba, "numba.decorators": dec, "streamlines": pkg, "streamlines.core": core})
    try:
        path = os.path.join(ref, "python", "streamlines", "preprocess.py")
        spec = importlib.util.spec_from_file_location("reference_preprocess", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v

    class NumbaTypedNumpy(types.ModuleType):
        """numpy, with np.hypot of integer scalars on float32."""

        def __getattr__(self, name):
            return getattr(np, name)

        @staticmethod
        def hypot(a, b, *args, **kw):
            if isinstance(a, np.integer) and isinstance(b, np.integer):
                return np.hypot(np.float32(a), np.float32(b))
            return np.hypot(a, b, *args, **kw)

        @staticmethod
        def dot(a, b, *args, **kw):
            if a is b:  # the speed of the mean velocity
                return np.dot(np.asarray(a, np.float64), np.asarray(b, np.float64))
            return np.dot(a, b, *args, **kw)
    mod.np = NumbaTypedNumpy("numpy_numba_typed")
    return mod


def make_roi(nx, ny, seed, noise, holes=False, dtype="float32", plateaus=False, pits=False, flat=False, **_):
    rng = np.random.default_rng(seed)
    if flat:
        roi = np.full((nx, ny), 50.0, dtype)
        roi[nx // 2, ny // 3] = 49.0
        roi[3, ny - 4] = np.nan
        return roi
    x = np.arange(nx)[:, None]
    y = np.arange(ny)[None, :]
    roi = 40.0 + 0.35 * x + 0.2 * y + 3.0 * np.sin(x / 5.0) * np.cos(y / 7.0)
    roi = roi + noise * rng.standard_normal((nx, ny))
    if pits:
        for _ in range(12):
            cx, cy = rng.integers(3, nx - 3), rng.integers(3, ny - 3)
            roi[cx - 1:cx + 2, cy - 1:cy + 2] -= 4.0 * rng.random()
    if plateaus:
        roi = np.round(roi * 2.0) / 2.0
    roi = roi.astype(dtype)
    if holes:
        roi[rng.random((nx, ny)) < 0.03] = np.nan
    return roi


def run_case(mod, nx, ny, seed, pixel_size, pad, noise, normalize=True, **kw):
    roi = make_roi(nx, ny, seed, noise, **kw)
    masks = []
    geodata = types.SimpleNamespace(
        roi_array=roi, pixel_size=float(pixel_size), pad_width=pad, roi_nx=nx, roi_ny=ny,
        x_roi_n_pixel_centers=np.linspace(0.5, nx - 1.5, nx - 1, dtype=np.float32),
        y_roi_n_pixel_centers=np.linspace(0.5, ny - 1.5, ny - 1, dtype=np.float32),
        dtm_mask_array=np.zeros((nx + 2 * pad, ny + 2 * pad), bool))
    state = types.SimpleNamespace(verbose=False, noisy=False,
                                  add_active_mask=lambda d: masks.append(d))
    P = mod.Preprocess
    me = P.__new__(P)  # the reference's Core.__init__ only copies parameters
    me.__dict__.update(geodata=geodata, state=state, print=lambda *a, **k: None,
                       vecsum_threshold=np.float64(0.95), divergence_threshold=np.float64(-0.5),
                       curl_threshold=np.float64(0.0), do_normalize_speed=normalize)
    me.conditioned_gradient_vector_field()
    me.mask_nan_uv()
    return dict(roi=roi, pixel_size=np.float64(pixel_size), pad_width=np.int64(pad),
                do_normalize_speed=np.bool_(normalize),
                uv_array=me.uv_array, slope_array=me.slope_array, uv_mask_array=masks[0]["uv"],
                blockages_array=me.blockages_array, blocked_neighbors_array=me.blocked_neighbors_array,
                where_looped_array=np.asarray(me.where_looped_array, np.uint32), n_loops=np.int64(me.n_loops),
                roi_gradx_array=me.roi_gradx_array, roi_grady_array=me.roi_grady_array)


def main():
    import warnings
    warnings.simplefilter("ignore", DeprecationWarning)
    mod = load_reference_preprocess(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_REF)
    for name, case in CASES.items():
        out = run_case(mod, **case)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "loops", int(out["n_loops"]), "blockages", int(np.count_nonzero(out["blockages_array"])),
              "blocked neighbours", int(np.count_nonzero(out["blocked_neighbors_array"])),
              "nan", int(out["uv_mask_array"].sum()))


if __name__ == "__main__":
    main()
