"""The reference's IndianCreek Test#2 job on its own real DTM (test helper).

tests/golden/indiancreek_test2.npz holds the job's region of interest (the
200 x 200 1 m DTM, x-major, no-data as NaN) and its basin mask (basins 1131
and 1132 kept), made from the reference's data/*.tif by
tests/golden/make_indiancreek_golden.py.

The reference's notebook tests/IndianCreek_Test2.ipynb recorded what its
stages found on this job (2018, the reference at commit 9da641c):

* preprocess (cell 12): 62 blockages;
* trace (cell 15): 15930 field seeds (the unmasked pixels) and the
  trajectory statistics of its 1000 seeds, in NOTEBOOK_STATS below.

The step counts n of the current reference kernels reproduce the notebook's
exactly.  The current kernels' trajectory length adds the Euler tail step's
raw distance to the clamped grid edge (rungekutta.cl:107-124), which the
2018 code did not; the notebook's l (and ds = l/n) is the sum of the
recorded steps, so l and ds are compared through the recorded steps.
"""
import os
import types

import numpy as np

from slm_b200.params import kernel_params
from slm_b200.useful import Data, Info, default_parameters, get_bbox

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "indiancreek_test2.npz")
PAD = 2
N_BLOCKAGES = 62
N_FIELD_SEEDS = 15930
# (direction, statistic) -> (l, n, ds), tests/IndianCreek_Test2.ipynb cell 15
NOTEBOOK_STATS = {
    ("downstream", "min"): (0.509221, 2.0, 0.254611),
    ("downstream", "mean"): (109.832016, 243.791, 0.448446),
    ("downstream", "max"): (253.752243, 563.0, 0.458204),
    ("upstream", "min"): (1.288012, 2.0, 0.265032),
    ("upstream", "mean"): (53.669567, 117.508003, 0.463404),
    ("upstream", "max"): (914.394592, 2000.0, 0.778504),
}
# relative tolerance of l and ds (recorded steps) against the notebook, per
# direction: downstream agrees to float32 summation order; upstream trajectories
# end through the Euler tail more often, which changed since 2018
L_DS_RTOL = {"downstream": 2e-5, "upstream": 2e-3}


def load():
    g = np.load(GOLDEN)
    return g["roi"], g["basin_mask"], float(g["pixel_size"])


def masks(roi, basin_mask, uv_mask):
    """The merged active mask of the job: dtm (NaN), basin and uv masks, padded."""
    dtm = np.pad(np.isnan(roi), PAD, constant_values=True)
    basin = np.pad(basin_mask, PAD, constant_values=True)
    return dtm | basin | uv_mask


def trace_inputs(mask, uv, pixel_size):
    """Info and the cropped Data of the Trace stage (trace.py:93-128), with the
    job's trace parameters (json/defaults.json: RK2, step 0.5 px, 1000
    trajectory seeds, d=3)."""
    d = default_parameters()
    bbox, nx, ny = get_bbox(~mask)
    info = Info(d.state, d.trace, pixel_size)
    info.set_xy(nx, ny, PAD)
    data = Data(info=info, bbox=bbox, pad=PAD, mapping_array=np.zeros(mask.shape, np.uint32),
                mask_array=mask, uv_array=uv)
    return info, data


def recorded_l_ds(steps_list, resolution=128):
    """Per trajectory: the sum of the recorded step lengths, and that over n."""
    res = np.float32(resolution)
    ls, ds = [], []
    for st in steps_list:
        v = st.astype(np.float32) / res
        l_ = float(np.sum(np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1]))) if len(st) else 0.0
        ls.append(l_)
        ds.append(l_ / len(st) if len(st) else np.nan)
    return np.array(ls), np.array(ds)


def check_stats(nsteps, steps_lists):
    """nsteps [n][2]; steps_lists[direction]: the recorded int8 (k, 2) steps
    of each trajectory.  Step counts as the notebook's (min, max exact; the
    mean to its 6 printed digits); the means of l and ds, and downstream the
    extremes of ds, within L_DS_RTOL.  Returns the values compared."""
    got = {}
    for col, name in enumerate(("downstream", "upstream")):
        n = nsteps[:, col].astype(np.float64)
        want = {k[1]: v for k, v in NOTEBOOK_STATS.items() if k[0] == name}
        assert n.min() == want["min"][1] and n.max() == want["max"][1], (name, n.min(), n.max())
        assert abs(n.mean() - want["mean"][1]) < 5e-4, (name, n.mean())
        ls, ds = recorded_l_ds(steps_lists[col])
        rtol = L_DS_RTOL[name]
        assert abs(ls.mean() / want["mean"][0] - 1) <= rtol, (name, ls.mean())
        assert abs(np.nanmean(ds) / want["mean"][2] - 1) <= rtol, (name, np.nanmean(ds))
        if name == "downstream":
            assert abs(np.nanmax(ds) / want["max"][2] - 1) <= rtol, (name, np.nanmax(ds))
            assert abs(np.nanmin(ds) / want["min"][2] - 1) <= rtol, (name, np.nanmin(ds))
        got[name] = {"n": (n.min(), n.mean(), n.max()), "l_mean": ls.mean(), "ds_mean": np.nanmean(ds),
                     "ds_min_max": (np.nanmin(ds), np.nanmax(ds))}
    return got


def state_for(mask):
    d = default_parameters()
    state = types.SimpleNamespace(**vars(d.state))
    state.merge_active_masks = lambda: mask.copy()
    return state


def field_params(info, sign):
    return kernel_params(info, "INTEGRATE_FIELDS", sign)
