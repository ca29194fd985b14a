"""Parity oracle -- TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the reference's kernels, both used only by
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference arms, and only as the checker or the baseline:

* the C restatement in this folder (``slm_oracle_*.c`` -> ``liboracle_slm.so``),
  which travels with the repository and is what the GPU parity tests compare
  against;
* the reference's own OpenCL C compiled on the host (``build_ref.py`` ->
  ``_ref/libref_<kernel>.so``), which pins the restatement: tests in this
  container check the restatement against it and ``tests/golden/`` holds
  vectors it produced.

Arrays are NumPy; the parameter block is ``slm_b200.params.SlmParams``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "liboracle_slm.so")
SOURCES = ["slm_oracle_trace.c", "slm_oracle_kde.c", "slm_oracle_map.c"]
REF_DIR = os.path.join(HERE, "_ref")

# mapping kernel -> number of buffer arguments after (params, seeds, n)
MAP_KERNELS = {
    "connect_channels": 3, "map_channel_heads": 3, "prune_channel_heads": 3,
    "count_downchannels": 5, "flag_downchannels": 5, "label_confluences": 6,
    "segment_downchannels": 6, "segment_hillslopes": 6, "subsegment_channel_edges": 6,
    "subsegment_flanks": 6, "fix_right_flanks": 6, "fix_left_flanks": 6,
    "hillslopes": 5, "hillslope_lengths": 5,
}

_lock = threading.Lock()
_lib = None


def build(force=False):
    """Compile the C restatement (gcc, OpenMP, strict IEEE binary32)."""
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    hdr = os.path.join(ROOT, "include", "slm_b200.h")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= max(os.path.getmtime(f) for f in srcs + [hdr])):
        return LIB_PATH
    cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-I", os.path.join(ROOT, "include")] + srcs + ["-o", LIB_PATH, "-lm"]
    subprocess.run(cmd, check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                build()
            L = ctypes.CDLL(LIB_PATH)
            P = ctypes.c_void_p
            u32, i32, u64 = ctypes.c_uint32, ctypes.c_int, ctypes.c_uint64
            L.oracle_integrate_fields.restype = u64
            L.oracle_integrate_fields.argtypes = [P, i32, P, u32, u32, u32, P, P, P, P, P, i32]
            L.oracle_field_seed_steps.restype = None
            L.oracle_field_seed_steps.argtypes = [P, i32, P, P, P, P, P, P, i32]
            L.oracle_integrate_trajectory.restype = u64
            L.oracle_integrate_trajectory.argtypes = [P, i32, u32, P, P, P, P, P, P, i32]
            for name in ("oracle_histogram_univariate", "oracle_histogram_bivariate"):
                getattr(L, name).restype = None
                getattr(L, name).argtypes = [P, P, u32, P]
            for name in ("oracle_pdf_univariate", "oracle_pdf_bivariate_rows",
                         "oracle_pdf_bivariate_cols"):
                getattr(L, name).restype = None
                getattr(L, name).argtypes = [P, P, P]
            for name, nargs in MAP_KERNELS.items():
                fn = getattr(L, "oracle_" + name)
                fn.restype = u32
                fn.argtypes = [P, P, u32] + [P] * nargs
            L.oracle_flank_paths.restype = u64
            L.oracle_flank_paths.argtypes = [P, P, u32, P, P, P, u32, P, P]
            _lib = L
        return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _params_ptr(p):
    return ctypes.cast(ctypes.byref(p), ctypes.c_void_p)


def _grid_inputs(seeds, mask, uv):
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    mask = np.ascontiguousarray(mask).view(np.uint8) if mask.dtype == np.bool_ else \
        np.ascontiguousarray(mask, dtype=np.uint8)
    uv = np.ascontiguousarray(uv, dtype=np.float32)
    return seeds, mask, uv


def integrate_fields(params, seeds, mask, uv, integrator=2, seed_begin=0, seed_end=None,
                     seed_stride=1, n_threads=1, slc=None, slt=None):
    """Restatement of integrate_fields; returns (slc u64, slt u64, steps, n_traj)."""
    seeds, mask, uv = _grid_inputs(seeds, mask, uv)
    nxy = params.nxy_padded
    if slc is None:
        slc = np.zeros(nxy, dtype=np.uint64)
    if slt is None:
        slt = np.zeros(nxy, dtype=np.uint64)
    ntraj = ctypes.c_uint64(0)
    end = params.n_seed_points if seed_end is None else seed_end
    steps = lib().oracle_integrate_fields(
        _params_ptr(params), integrator, _ptr(seeds), seed_begin, end, seed_stride,
        _ptr(mask), _ptr(uv), _ptr(slc), _ptr(slt),
        ctypes.cast(ctypes.byref(ntraj), ctypes.c_void_p), n_threads)
    return slc, slt, int(steps), int(ntraj.value)


def field_seed_steps(params, seeds, mask, uv, integrator=2, n_threads=1):
    """Per-seed RK step counts (uint32 [n_seed_points], the sum over each seed's
    d*d trajectories) of a field pass of the restatement."""
    seeds, mask, uv = _grid_inputs(seeds, mask, uv)
    nxy = params.nxy_padded
    slc = np.zeros(nxy, dtype=np.uint64)
    slt = np.zeros(nxy, dtype=np.uint64)
    out = np.zeros(int(params.n_seed_points), dtype=np.uint32)
    lib().oracle_field_seed_steps(_params_ptr(params), integrator, _ptr(seeds), _ptr(mask), _ptr(uv),
                                  _ptr(slc), _ptr(slt), _ptr(out), n_threads)
    return out


def integrate_trajectory(params, n_chunk, seeds, mask, uv, integrator=2, n_threads=1):
    """Restatement of integrate_trajectory; returns (traj int8 [n_chunk,max_n_steps,2],
    nsteps u16, length f32, steps)."""
    seeds, mask, uv = _grid_inputs(seeds, mask, uv)
    traj = np.zeros((n_chunk, params.max_n_steps, 2), dtype=np.int8)
    nsteps = np.zeros(n_chunk, dtype=np.uint16)
    length = np.zeros(n_chunk, dtype=np.float32)
    steps = lib().oracle_integrate_trajectory(
        _params_ptr(params), integrator, n_chunk, _ptr(seeds), _ptr(mask), _ptr(uv),
        _ptr(traj), _ptr(nsteps), _ptr(length), n_threads)
    return traj, nsteps, length, int(steps)


# ------------------------------------------------------------------ reference arm
class RefKernel:
    """One reference kernel compiled on the host (``_ref/libref_<name>.so``)."""

    _cache = {}

    def __init__(self, name):
        path = os.path.join(REF_DIR, "libref_{}.so".format(name))
        if not os.path.exists(path):
            raise FileNotFoundError(
                "{} missing: build it with oracle/build_ref.py where the reference "
                "checkout is present".format(path))
        self.lib = ctypes.CDLL(path)
        self.lib.slmref_run.restype = ctypes.c_int
        self.lib.slmref_run.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_int]
        from slm_b200.params import SlmParams
        self.P = SlmParams.in_dll(self.lib, "slmref_P")

    @classmethod
    def get(cls, name):
        if name not in cls._cache:
            cls._cache[name] = cls(name)
        return cls._cache[name]

    def run(self, params, arrays, n_global, offset=0, n_threads=1):
        ctypes.memmove(ctypes.byref(self.P), ctypes.byref(params), ctypes.sizeof(self.P))
        argv = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
        self.lib.slmref_run(argv, n_global, offset, n_threads)


def ref_available(name="integrate_fields"):
    return os.path.exists(os.path.join(REF_DIR, "libref_{}.so".format(name)))


def ref_integrate_fields(params, seeds, mask, uv, n_threads=1, n_global=None):
    """The reference kernel itself; returns (slc u32, slt u32) as the reference keeps them."""
    seeds, mask, uv = _grid_inputs(seeds, mask, uv)
    nxy = params.nxy_padded
    mapping = np.zeros(nxy, dtype=np.uint32)
    slc = np.zeros(nxy, dtype=np.uint32)
    slt = np.zeros(nxy, dtype=np.uint32)
    n = params.n_seed_points if n_global is None else n_global
    RefKernel.get("integrate_fields").run(params, [seeds, mask, uv, mapping, slc, slt], n,
                                          0, n_threads)
    return slc, slt


def ref_integrate_trajectory(params, n_chunk, seeds, mask, uv, n_threads=1):
    seeds, mask, uv = _grid_inputs(seeds, mask, uv)
    mapping = np.zeros(params.nxy_padded, dtype=np.uint32)
    traj = np.zeros((n_chunk, params.max_n_steps, 2), dtype=np.int8)
    nsteps = np.zeros(n_chunk, dtype=np.uint16)
    length = np.zeros(n_chunk, dtype=np.float32)
    RefKernel.get("integrate_trajectory").run(
        params, [seeds, mask, uv, mapping, traj, nsteps, length], n_chunk, 0, n_threads)
    return traj, nsteps, length


# ------------------------------------------------------------------ KDE
KDF_SHAPES = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]


def histogram_univariate(params, data):
    data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1)
    hist = np.zeros(params.n_hist_bins, dtype=np.uint32)
    lib().oracle_histogram_univariate(_params_ptr(params), _ptr(data), data.size, _ptr(hist))
    return hist


def histogram_bivariate(params, data):
    data = np.ascontiguousarray(data, dtype=np.float32).reshape(-1, 2)
    hist = np.zeros(params.n_hist_bins * params.n_hist_bins, dtype=np.uint32)
    lib().oracle_histogram_bivariate(_params_ptr(params), _ptr(data), data.shape[0], _ptr(hist))
    return hist


def pdf_univariate(params, hist):
    hist = np.ascontiguousarray(hist, dtype=np.uint32).reshape(-1)
    pdf = np.zeros(params.n_pdf_points, dtype=np.float32)
    lib().oracle_pdf_univariate(_params_ptr(params), _ptr(hist), _ptr(pdf))
    return pdf


def pdf_bivariate_rows(params, hist):
    hist = np.ascontiguousarray(hist, dtype=np.uint32).reshape(-1)
    out = np.zeros(params.n_hist_bins * params.n_hist_bins, dtype=np.float32)
    lib().oracle_pdf_bivariate_rows(_params_ptr(params), _ptr(hist), _ptr(out))
    return out


def pdf_bivariate_cols(params, partial):
    partial = np.ascontiguousarray(partial, dtype=np.float32).reshape(-1)
    out = np.zeros(params.n_pdf_points * params.n_pdf_points, dtype=np.float32)
    lib().oracle_pdf_bivariate_cols(_params_ptr(params), _ptr(partial), _ptr(out))
    return out


def ref_kde(name, params, inp, out_size, out_dtype, n_global):
    """Run one reference KDE kernel (pdf kernels pick the KDF_IS_<shape> build)."""
    if name.startswith("pdf_"):
        name = "{}__{}".format(name, KDF_SHAPES[params.kdf_kind])
    out = np.zeros(out_size, dtype=out_dtype)
    RefKernel.get(name).run(params, [np.ascontiguousarray(inp), out], n_global, 0, 1)
    return out


# ------------------------------------------------------------------ mapping
def map_kernel(name, params, seeds, arrays):
    """Run one mapping kernel of the restatement in place on ``arrays`` (the
    reference kernel's buffers after seed_point, in order); returns the status
    word (bit 0 loop cap hit, bit 1 out-of-grid access skipped)."""
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    fn = getattr(lib(), "oracle_" + name)
    ptrs = []
    for a in arrays:
        assert a.flags["C_CONTIGUOUS"], name
        ptrs.append(ctypes.c_void_p(a.ctypes.data))
    return int(fn(_params_ptr(params), _ptr(seeds), seeds.shape[0], *ptrs))


def ref_map_kernel(name, params, seeds, arrays):
    """The reference's own mapping kernel, sequential ascending global id, in place."""
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    p = params.copy()
    p.n_seed_points = seeds.shape[0]
    RefKernel.get(name).run(p, [seeds] + list(arrays), seeds.shape[0], 0, 1)


def flank_paths(params, seeds, mask, uv, mapping, cap=4096):
    """(counts [n], pairs [n, cap, 2]) of the flank walks (tests only)."""
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    n = seeds.shape[0]
    counts = np.zeros(n, dtype=np.uint32)
    pairs = np.zeros((n, cap, 2), dtype=np.uint32)
    lib().oracle_flank_paths(_params_ptr(params), _ptr(seeds), n,
                             _ptr(np.ascontiguousarray(mask).view(np.uint8)), _ptr(uv),
                             _ptr(mapping), cap, _ptr(counts), _ptr(pairs))
    return counts, pairs
