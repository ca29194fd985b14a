"""Kernel parameter block shared by every C-ABI entry point.

The reference passes every scalar to its OpenCL kernels as a ``-D NAME=value``
macro produced by ``pocl.set_compile_options`` (reference
``python/streamlines/pocl.py:178-299``) and rebuilds the program for each
distinct set.  Here the same values travel at run time in one POD struct,
``slm_params`` (``include/slm_b200.h``), whose fields are the macros' names in
lower case.  ``compile_options`` restates the reference's macro derivation
(same names, same values, same string formatting), and ``params_from_options``
turns such a list into the struct the way a C compiler reads the macros: a
``u`` literal is an unsigned 32-bit integer (so ``-1u`` is 4294967295) and an
``f`` literal is parsed by ``strtof`` (correctly rounded to binary32).
"""
from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

# (field, kind) in struct order; kind 'u' = uint32, 'f' = float32.
FIELDS = [
    # integration macros, pocl.py:231-277
    ("n_seed_points", "u"), ("downup_sign", "u"),
    ("integrator_step_factor", "f"), ("max_integration_step_error", "f"),
    ("adjusted_max_error", "f"), ("integration_halt_threshold", "f"),
    ("max_length", "f"), ("pixel_size", "f"),
    ("pad_width", "u"), ("pad_width_pp5", "f"),
    ("nx_padded", "u"), ("ny_padded", "u"), ("nxy_padded", "u"),
    ("nxf_mp5", "f"), ("nyf_mp5", "f"), ("grid_scale", "f"),
    ("combo_factor", "f"), ("dt_max", "f"),
    ("max_n_steps", "u"), ("trajectory_resolution", "u"),
    ("seeds_chunk_offset", "u"), ("subpixel_seed_point_density", "u"),
    ("subpixel_seed_halfspan", "f"), ("subpixel_seed_step", "f"),
    ("jitter_magnitude", "f"),
    ("interchannel_max_n_steps", "u"), ("left_flank_addition", "u"),
    ("is_channel", "u"), ("is_thinchannel", "u"), ("is_interchannel", "u"),
    ("is_channelhead", "u"), ("is_channeltail", "u"),
    ("is_majorconfluence", "u"), ("is_minorconfluence", "u"),
    ("is_majorinflow", "u"), ("is_minorinflow", "u"),
    ("is_leftflank", "u"), ("is_rightflank", "u"),
    ("is_midslope", "u"), ("is_ridge", "u"), ("was_channelhead", "u"),
    ("is_subsegmenthead", "u"), ("is_loop", "u"), ("is_blockage", "u"),
    ("segmentation_threshold", "u"),
    # kde macros, pocl.py:197-217
    ("bandwidth", "f"), ("n_data", "u"), ("n_hist_bins", "u"), ("n_pdf_points", "u"),
    ("logx_min", "f"), ("logx_max", "f"), ("logx_range", "f"),
    ("bin_dx", "f"), ("pdf_dx", "f"), ("kdf_width_x", "f"),
    ("n_kdf_part_points_x", "u"),
    ("logy_min", "f"), ("logy_max", "f"), ("logy_range", "f"),
    ("bin_dy", "f"), ("pdf_dy", "f"), ("kdf_width_y", "f"),
    ("n_kdf_part_points_y", "u"),
    # flags (0/1): DO_MEASURE_HSL_FROM_RIDGES and the KDF_IS_<SHAPE> selector
    ("do_measure_hsl_from_ridges", "u"), ("kdf_kind", "u"),
]

FIELD_NAMES = [f for f, _ in FIELDS]

# KDF_IS_<shape> selector values carried in slm_params.kdf_kind
KDF_KINDS = {"tophat": 0, "triangle": 1, "epanechnikov": 2, "cosine": 3, "gaussian": 4}


class SlmParams(ctypes.Structure):
    """ctypes mirror of ``slm_params`` in ``include/slm_b200.h``."""
    _fields_ = [(n, ctypes.c_uint32 if k == "u" else ctypes.c_float) for n, k in FIELDS]

    def as_dict(self):
        return {n: getattr(self, n) for n in FIELD_NAMES}

    def copy(self):
        c = SlmParams()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(SlmParams))
        return c


_libc = ctypes.CDLL(ctypes.util.find_library("c") or None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]


def strtof(text: str) -> float:
    """Parse a decimal literal to binary32 with correct rounding (C ``strtof``)."""
    return float(np.float32(_libc.strtof(text.encode(), None)))


# The integration macro table of pocl.set_compile_options (pocl.py:231-277):
# name -> (literal suffix, override-or-'').  Entries whose override is '' take
# getattr(info, name).  Order matters only for the emitted option list.
def _integration_table(info, downup_sign):
    pad = np.uint32(info.pad_width)
    nxp = np.uint32(info.nx_padded)
    nyp = np.uint32(info.ny_padded)
    nxf = np.float32(info.nx)
    nyf = np.float32(info.ny)
    grid_scale = np.float32(np.sqrt(nxf * nyf))
    combo_factor = np.float32(grid_scale * info.integrator_step_factor)
    dt_max = np.float32(min(min(1.0 / nxf, 1.0 / nyf), 0.1))
    table = {
        "n_seed_points": ("u", ""),
        "downup_sign": ("u", np.int8(downup_sign)),
        "integrator_step_factor": ("f", ""),
        "max_integration_step_error": ("f", ""),
        "adjusted_max_error": ("f", ""),
        "integration_halt_threshold": ("f", ""),
        "max_length": ("f", ""),
        "pixel_size": ("f", ""),
        "pad_width": ("u", pad),
        "pad_width_pp5": ("f", np.float32(pad) + 0.5),
        "nx_padded": ("u", nxp),
        "ny_padded": ("u", nyp),
        "nxy_padded": ("u", np.uint32(nxp * nyp)),
        "nxf_mp5": ("f", nxf - 0.5),
        "nyf_mp5": ("f", nyf - 0.5),
        "grid_scale": ("f", grid_scale),
        "combo_factor": ("f", combo_factor * downup_sign),
        "dt_max": ("f", dt_max),
        "max_n_steps": ("u", ""),
        "trajectory_resolution": ("u", ""),
        "seeds_chunk_offset": ("u", ""),
        "subpixel_seed_point_density": ("u", ""),
        "subpixel_seed_halfspan": ("f", ""),
        "subpixel_seed_step": ("f", ""),
        "jitter_magnitude": ("f", ""),
        "interchannel_max_n_steps": ("u", ""),
        "left_flank_addition": ("u", ""),
    }
    for flag in ("is_channel", "is_thinchannel", "is_interchannel", "is_channelhead",
                 "is_channeltail", "is_majorconfluence", "is_minorconfluence",
                 "is_majorinflow", "is_minorinflow", "is_leftflank", "is_rightflank",
                 "is_midslope", "is_ridge", "was_channelhead", "is_subsegmenthead",
                 "is_loop", "is_blockage"):
        table[flag] = ("u", "")
    table["do_measure_hsl_from_ridges"] = ("flag", "")
    table["debug"] = ("flag", "")
    table["verbose"] = ("flag", "")
    if info.segmentation_threshold > 0:
        table["segmentation_threshold"] = ("u", "")
    return table


_KDE_TABLE = [
    ("bandwidth", "f"), ("n_data", "u"), ("n_hist_bins", "u"), ("n_pdf_points", "u"),
    ("logx_min", "f"), ("logx_max", "f"), ("logx_range", "f"), ("bin_dx", "f"),
    ("pdf_dx", "f"), ("kdf_width_x", "f"), ("n_kdf_part_points_x", "u"),
    ("logy_min", "f"), ("logy_max", "f"), ("logy_range", "f"), ("bin_dy", "f"),
    ("pdf_dy", "f"), ("kdf_width_y", "f"), ("n_kdf_part_points_y", "u"),
]


def compile_options(info, kernel_def, downup_sign=1, job_type="integration"):
    """The ``-D`` option list the reference builds for ``kernel_def``.

    Restates ``pocl.set_compile_options`` (pocl.py:178-299) value for value,
    including its handling of false flags, which repeats the previous entry.
    """
    rtn = ["-D", "KERNEL_{}".format(kernel_def.upper())]
    if job_type == "kde":
        rtn += ["-D", "KDF_IS_{}".format(info.kernel.upper())]
        for name, suffix in _KDE_TABLE:
            rtn += ["-D", "{0}={1}{2}".format(name.upper(), getattr(info, name), suffix)]
        return rtn
    item = None
    for name, (suffix, override) in _integration_table(info, downup_sign).items():
        if suffix == "flag":
            if getattr(info, name):
                item = ["-D", "{}".format(name.upper())]
        elif not (isinstance(override, str) and override == ""):
            item = ["-D", "{0}={1}{2}".format(name.upper(), override, suffix)]
        else:
            item = ["-D", "{0}={1}{2}".format(name.upper(), getattr(info, name), suffix)]
        rtn += item
    return rtn


def params_from_options(options) -> SlmParams:
    """Read a ``-D`` option list the way the OpenCL C compiler reads the macros."""
    p = SlmParams()
    kinds = dict(FIELDS)
    defines = [options[i + 1] for i in range(0, len(options), 2) if options[i] == "-D"]
    for d in defines:
        if "=" not in d:
            if d.startswith("KDF_IS_"):
                p.kdf_kind = KDF_KINDS[d[len("KDF_IS_"):].lower()]
            elif d == "DO_MEASURE_HSL_FROM_RIDGES":
                p.do_measure_hsl_from_ridges = 1
            continue
        name, lit = d.split("=", 1)
        field = name.lower()
        if field not in kinds:
            continue
        if lit.endswith("u"):
            setattr(p, field, int(lit[:-1]) & 0xFFFFFFFF)
        elif lit.endswith("f"):
            setattr(p, field, strtof(lit[:-1]))
        else:
            raise ValueError("unexpected macro literal {!r}".format(d))
    return p


def kernel_params(info, kernel_def="INTEGRATE_FIELDS", downup_sign=1, job_type="integration"):
    """Parameter block for one launch (what the reference compiles in as macros)."""
    return params_from_options(compile_options(info, kernel_def, downup_sign, job_type))
