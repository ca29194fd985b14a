"""The Trace stage mirror against the reference's own Trace class (CPU only).

Both run with the same CPU stand-ins for Trajectories and Fields, whose
outputs depend on the cropped arrays they are handed; the comparison covers
what Trace itself does (trace.py:93-170): the bounding-box crop of the merged
mask and of uv, the trajectory seeds' offset back to the ROI frame, and the
write-back of the fields into full padded arrays with slc truncated to
uint32."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

from slm_b200 import trace as T
from slm_b200.useful import default_parameters
from test_params import _load_reference_modules


class FakeTrajectories:
    def __init__(self, cl_platform, cl_device, cl_src_path=None, info=None, data=None, do_trace_downstream=True,
                 do_trace_upstream=True, verbose=False, gpu_verbose=False, integrator=2):
        self.data = data

    def integrate(self):
        d = self.data
        d.seed_point_array = np.argwhere(~d.mask_array).astype(np.float32)[:9] + np.float32(0.25)
        d.streamline_arrays_list = [[np.arange(4, dtype=np.int8)], [np.arange(3, dtype=np.int8)]]
        d.traj_stats_df = ("stats", d.mask_array.shape)


class FakeFields:
    def __init__(self, cl_platform, cl_device, cl_src_path=None, info=None, data=None, verbose=False,
                 gpu_verbose=False, schedule="persistent", integrator=2):
        self.data = data

    def prepare(self, trace=True):
        pass

    def integrate(self):
        d = self.data
        u = d.uv_array.astype(np.float64)
        d.slc_array = np.abs(u) * 37.3 + 0.9  # fractional: the uint32 store truncates
        d.slt_array = (u * 5.5).astype(np.float32)
        d.sla_array = (u[:, :, ::-1] * 2.25).astype(np.float32)


def _reference_trace(reference_dir):
    mods = _load_reference_modules(reference_dir)
    stub = {"streamlines.core": types.ModuleType("streamlines.core"),
            "streamlines.trajectories": types.ModuleType("streamlines.trajectories"),
            "streamlines.fields": types.ModuleType("streamlines.fields")}

    class Core:
        def __init__(self, state, imported_parameters):
            self.state = state
            for k, v in imported_parameters["trace"].items():
                setattr(self, k, v)

        def print(self, *a, **k):
            pass
    stub["streamlines.core"].Core = Core
    stub["streamlines.trajectories"].Trajectories = FakeTrajectories
    stub["streamlines.fields"].Fields = FakeFields
    pkg = types.ModuleType("streamlines")
    keys = list(stub) + ["streamlines", "streamlines.useful"]
    saved = {k: sys.modules.get(k) for k in keys}
    sys.modules.update(stub)
    sys.modules["streamlines"] = pkg
    sys.modules["streamlines.useful"] = mods["useful"]
    try:
        spec = importlib.util.spec_from_file_location(
            "reference_trace", os.path.join(reference_dir, "python", "streamlines", "trace.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_trace_stage_matches_reference(reference_dir, seed, monkeypatch):
    R = _reference_trace(reference_dir)
    rng = np.random.default_rng(seed)
    nx, ny, pad = 40 + seed * 7, 33 + seed * 5, 2
    mask = np.ones((nx + 2 * pad, ny + 2 * pad), bool)
    x0, y0 = pad + 3 + seed, pad + 2 * seed
    mask[x0:pad + nx - 4, y0:pad + ny - 1 - seed] = False  # the unmasked region: a smaller box
    mask[x0 + 5, y0 + 3] = True
    uv = rng.standard_normal((nx + 2 * pad, ny + 2 * pad, 2)).astype(np.float32)
    d = default_parameters()
    state = types.SimpleNamespace(**vars(d.state))
    state.merge_active_masks = lambda: mask.copy()
    state.cl_src_path = None
    params = {"trace": dict(vars(d.trace))}
    geodata = types.SimpleNamespace(roi_nx=nx, roi_ny=ny, pad_width=pad, roi_pixel_size=1.0)
    preprocess = types.SimpleNamespace(uv_array=uv)
    ref = R.Trace(state, params, geodata, preprocess)
    ref.do()
    monkeypatch.setattr(T, "Trajectories", FakeTrajectories)
    monkeypatch.setattr(T, "Fields", FakeFields)
    mine = T.Trace(state, params, geodata, preprocess)
    mine.do()
    assert np.array_equal(mine.seed_point_array, ref.seed_point_array)
    assert mine.seed_point_array.dtype == ref.seed_point_array.dtype
    assert mine.traj_stats_df == ref.traj_stats_df
    for k in ("slc_array", "slt_array", "sla_array"):
        a, b = getattr(mine, k), getattr(ref, k)
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b), k
    assert mine.slc_array.dtype == np.uint32 and mine.slc_array.any()
