"""map_midslopes / map_ridges against the reference's own methods (CPU only).

The reference's mapping.py is loaded with stand-ins for its GPU wrappers and
for scikit-image (absent here); both sides thin with this package's host
Zhang-Suen thinning, so the flags must agree exactly."""
import importlib.util
import os
import sys
import types

import numpy as np
import pytest

from slm_b200 import mapping as M
from slm_b200.skeleton import zhang_suen
from slm_b200.useful import Data, Info, default_parameters
from test_params import _load_reference_modules


def _reference_mapping(reference_dir):
    mods = _load_reference_modules(reference_dir)
    stub_names = ["skimage", "skimage.morphology", "skimage.filters", "skimage.filters.rank", "skfmm",
                  "streamlines", "streamlines.core", "streamlines.useful", "streamlines.pocl"] + \
        ["streamlines." + n for n in ("connect", "channelheads", "countlink", "label", "segment", "hillslopes",
                                      "lengths")]
    saved = {k: sys.modules.get(k) for k in stub_names}
    st = {k: types.ModuleType(k) for k in stub_names}
    st["skimage.morphology"].skeletonize = zhang_suen
    for n in ("thin", "medial_axis", "disk"):
        setattr(st["skimage.morphology"], n, None)
    st["skimage.filters"].gaussian = None
    st["skimage.filters.rank"].mean = st["skimage.filters.rank"].median = None
    st["streamlines.core"].Core = type("Core", (), {})
    st["streamlines.pocl"].Initialize_cl = None
    for n in ("connect", "channelheads", "countlink", "label", "segment", "hillslopes", "lengths"):
        setattr(st["streamlines"], n, st["streamlines." + n])
    sys.modules.update(st)
    sys.modules["streamlines.useful"] = mods["useful"]
    if not hasattr(np, "bool"):
        np.bool = np.bool_  # the reference's dtype=np.bool (NumPy < 1.24)
    try:
        spec = importlib.util.spec_from_file_location(
            "reference_mapping", os.path.join(reference_dir, "python", "streamlines", "mapping.py"))
        mod = importlib.util.module_from_spec(spec)
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            spec.loader.exec_module(mod)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    return mod


def _case(seed):
    rng = np.random.default_rng(seed)
    nx, ny = 70, 64
    d = default_parameters()
    info = Info(d.state, d.trace, 1.0, mapping=d.mapping)
    info.set_xy(nx, ny, 2)
    nxp, nyp = nx + 4, ny + 4
    x = np.linspace(0, 4, nxp)[:, None]
    y = np.linspace(0, 3, nyp)[None, :]
    base = np.exp(2.0 + np.sin(x * 2.1) * np.cos(y * 1.7))
    ridge_band = np.where(np.abs(np.arange(nxp) - 25 - 3 * seed) < 6, 0.04, 1.0)[:, None]  # dsla << usla
    sla = np.stack([base * ridge_band * (1 + 0.3 * rng.random((nxp, nyp))),
                    base[::-1] * (1 + 0.3 * rng.random((nxp, nyp)))], 2).astype(np.float32)
    mask = np.zeros((nxp, nyp), bool)
    mask[:2], mask[-2:], mask[:, :2], mask[:, -2:] = True, True, True, True
    mask[rng.random((nxp, nyp)) < 0.02] = True
    data = Data(info=info, mask_array=mask, uv_array=None, mapping_array=np.zeros((nxp, nyp), np.uint32),
                sla_array=sla)
    return info, data


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("what", ["midslopes", "ridges"])
def test_filters_match_reference(reference_dir, seed, what):
    R = _reference_mapping(reference_dir)
    info, data = _case(seed)
    ref = R.Mapping.__new__(R.Mapping)
    ref.__dict__.update(midslope_filter_sigma=5.0, midslope_threshold=0.03, ridge_filter_sigma=2.0,
                        ridge_threshold=0.8, print=lambda *a, **k: None)
    rdata = Data(info=info, mask_array=data.mask_array, uv_array=None, mapping_array=data.mapping_array,
                 sla_array=data.sla_array)
    if what == "midslopes":
        if not hasattr(np, "bool"):
            pytest.skip("NumPy without np.bool")
        R.Mapping.map_midslopes(ref, info, rdata)
        M.map_midslopes(info, data, 5.0, 0.03, thin=zhang_suen)
        flag = info.is_midslope
    else:
        R.Mapping.map_ridges(ref, info, rdata)
        M.map_ridges(info, data, 2.0, 0.8, thin=zhang_suen)
        flag = info.is_ridge
    assert np.array_equal(data.mapping_array, rdata.mapping_array)
    assert ((data.mapping_array & flag) > 0).sum() > 0
