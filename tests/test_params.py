"""Parameter derivation and the C struct layout (CPU only).

Where the reference checkout is present, its own ``pocl.set_compile_options``
and ``useful.Info`` are imported with stand-ins for the modules missing here
(pyopencl, GDAL, pympler) and compared with this package's restatements.
"""
import importlib.util
import os
import re
import sys
import types

import numpy as np
import pytest

from cases import Case
from slm_b200 import params as P
from slm_b200.useful import Info, default_parameters

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_reference_modules(reference_dir):
    """Import the reference's useful.py and pocl.py with import stand-ins."""
    saved = {k: sys.modules.get(k) for k in
             ("pyopencl", "pyopencl.tools", "osgeo", "pympler", "pympler.asizeof",
              "streamlines", "streamlines.useful")}
    try:
        cl = types.ModuleType("pyopencl")
        cl.tools = types.ModuleType("pyopencl.tools")
        sys.modules["pyopencl"] = cl
        sys.modules["pyopencl.tools"] = cl.tools
        osgeo = types.ModuleType("osgeo")
        osgeo.gdal = types.ModuleType("gdal")
        sys.modules["osgeo"] = osgeo
        pym = types.ModuleType("pympler")
        pym.asizeof = types.ModuleType("pympler.asizeof")
        pym.asizeof.asizeof = lambda x: 0
        sys.modules["pympler"] = pym
        sys.modules["pympler.asizeof"] = pym.asizeof
        if not hasattr(np, "bool8"):
            np.bool8 = np.bool_
        pkg = types.ModuleType("streamlines")
        pkg.__path__ = [os.path.join(reference_dir, "python", "streamlines")]
        sys.modules["streamlines"] = pkg
        mods = {}
        for name in ("useful", "pocl"):
            spec = importlib.util.spec_from_file_location(
                "streamlines." + name, os.path.join(reference_dir, "python", "streamlines", name + ".py"))
            m = importlib.util.module_from_spec(spec)
            sys.modules["streamlines." + name] = m
            spec.loader.exec_module(m)
            mods[name] = m
        return mods
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


@pytest.fixture(scope="module")
def ref_modules(reference_dir):
    return _load_reference_modules(reference_dir)


TRACE_VARIANTS = [
    dict(density=3, jitter=1.0, step=0.5, max_length=1000.0, pixel_size=1.0, nx=200, ny=200),
    dict(density=2, jitter=1.0, step=0.1, max_length=1000.0, pixel_size=2.0, nx=2048, ny=2048),
    dict(density=1, jitter=0.0, step=0.1, max_length=200.0, pixel_size=1.0, nx=512, ny=512),
    dict(density=2, jitter=1.0, step=0.1, max_length=2000.0, pixel_size=1.0, nx=8192, ny=8192),
    dict(density=3, jitter=1.0, step=0.5, max_length=30.0, pixel_size=2.0, nx=142, ny=240),
]


def _infos(ref_useful, v):
    d = default_parameters()
    d.trace.subpixel_seed_point_density = v["density"]
    d.trace.jitter_magnitude = v["jitter"]
    d.trace.integrator_step_factor = v["step"]
    d.trace.max_length = v["max_length"]
    mine = Info(d.state, d.trace, v["pixel_size"], mapping=d.mapping)
    mine.set_xy(v["nx"], v["ny"], 2)
    theirs = ref_useful.Info(d.state, d.trace, v["pixel_size"], mapping=d.mapping)
    theirs.set_xy(v["nx"], v["ny"], 2)
    for inf in (mine, theirs):
        inf.n_seed_points = np.uint32(1234)
    return mine, theirs


@pytest.mark.parametrize("v", TRACE_VARIANTS)
@pytest.mark.parametrize("kernel,sign", [("INTEGRATE_FIELDS", 1.0), ("INTEGRATE_FIELDS", -1.0),
                                         ("INTEGRATE_TRAJECTORY", np.float32(-1.0)),
                                         ("SEGMENT_DOWNCHANNELS", 1)])
def test_compile_options_match_reference(ref_modules, v, kernel, sign):
    mine, theirs = _infos(ref_modules["useful"], v)
    if kernel == "SEGMENT_DOWNCHANNELS":
        mine.set_thresholds(segmentation_threshold=np.uint32(10))
        theirs.set_thresholds(segmentation_threshold=np.uint32(10))
    ref = ref_modules["pocl"].set_compile_options(theirs, kernel, downup_sign=sign)
    assert P.compile_options(mine, kernel, sign) == ref


def test_kde_options_match_reference(ref_modules):
    info = types.SimpleNamespace(kernel="gaussian", bandwidth=np.float32(0.25),
                                 n_data=np.uint32(1000), n_hist_bins=np.uint32(2048),
                                 n_pdf_points=np.uint32(256), logx_min=np.float32(-1.5),
                                 logx_max=np.float32(3.25), logx_range=np.float32(4.75),
                                 bin_dx=np.float32(0.002), pdf_dx=np.float32(0.018),
                                 kdf_width_x=np.float32(0.3), n_kdf_part_points_x=np.uint32(17),
                                 logy_min=0, logy_max=0, logy_range=0, bin_dy=0, pdf_dy=0,
                                 kdf_width_y=0, n_kdf_part_points_y=0)
    ref = ref_modules["pocl"].set_compile_options(info, "pdf_univariate", job_type="kde")
    assert P.compile_options(info, "pdf_univariate", job_type="kde") == ref
    prm = P.params_from_options(ref)
    assert prm.kdf_kind == P.KDF_KINDS["gaussian"] and prm.n_hist_bins == 2048


def test_params_parse_like_c():
    c = Case()
    up = c.params("INTEGRATE_FIELDS", -1.0)
    down = c.params("INTEGRATE_FIELDS", 1.0)
    assert up.downup_sign == 0xFFFFFFFF and down.downup_sign == 1
    assert up.combo_factor == -down.combo_factor
    g = np.float32(np.sqrt(np.float32(40) * np.float32(56)))
    assert np.float32(down.grid_scale) == g
    assert np.float32(down.combo_factor) == np.float32(g * np.float32(0.5))
    assert down.nxy_padded == 44 * 60 and down.max_n_steps == 200
    assert P.strtof("0.1") == float(np.float32(0.1))


def _header_struct_fields():
    text = open(os.path.join(ROOT, "include", "slm_b200.h")).read()
    body = re.search(r"typedef struct slm_params \{(.*?)\} slm_params;", text, re.S).group(1)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(uint32_t|float)\s+(.*)", decl, re.S)
        assert m, decl
        kind = "u" if m.group(1) == "uint32_t" else "f"
        for n in m.group(2).split(","):
            names.append((n.strip(), kind))
    return names


def test_struct_layout_matches_header():
    assert _header_struct_fields() == P.FIELDS
    assert len(P.FIELDS) == len(set(P.FIELD_NAMES))


@pytest.mark.parametrize("shape,holes", [((30, 40), 0), ((257, 129), 40), ((64, 64), 4000)])
def test_create_seeds_matches_reference(ref_modules, shape, holes):
    from slm_b200.useful import create_seeds
    rng = np.random.default_rng(holes)
    mask = np.zeros(shape, dtype=bool)
    mask[:2, :] = mask[-2:, :] = mask[:, :2] = mask[:, -2:] = True
    if holes:
        mask[rng.integers(0, shape[0], holes), rng.integers(0, shape[1], holes)] = True
    for n_seed_points in (None, 17):
        for rng_seed in (1, 7):
            ref = ref_modules["useful"].create_seeds(mask, 2, 32, n_seed_points=n_seed_points,
                                                     do_shuffle=True, rng_seed=rng_seed)
            st_ref = np.random.get_state()[1].copy()
            for _ in range(2):  # second call is served from the cache
                mine = create_seeds(mask, 2, 32, n_seed_points=n_seed_points,
                                    do_shuffle=True, rng_seed=rng_seed)
                assert np.array_equal(ref[0], mine[0]) and ref[1:] == mine[1:]
                assert np.array_equal(np.random.get_state()[1], st_ref)
