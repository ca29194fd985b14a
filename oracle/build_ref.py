#!/usr/bin/env python3
"""Build the reference's own OpenCL kernels as host shared libraries.

TEST INFRASTRUCTURE ONLY.  Output goes to ``oracle/_ref/`` (git-ignored; the
built ``.so`` files travel with the repository snapshot to GPU hosts, where the
reference checkout is absent).

For every kernel the reference's Python wrapper builds, this script
concatenates the same ``opencl/*.cl`` files in the same order (the file lists
below cite the wrapper lines), prepends ``cl_shim.hpp`` and a ``#define`` of
every ``-D`` macro of ``pocl.set_compile_options`` as a field of a run-time
parameter struct (``slmref_P``, same layout as ``slm_params``), and compiles the
result with g++ (no FMA contraction, no fast-math).  Three syntactic rewrites
make OpenCL C parse as C++ without changing what it computes:

1. ``(float2)(a,b)`` / ``(char2)(a,b)`` vector literals -> ``float2{a,b}`` /
   ``char2{a,b}`` (braced init evaluates a then b, i.e. left to right);
2. ``(char)(x)`` -> ``slm_cvt_char(x)`` (x86 truncation, see cl_shim.hpp);
3. connect_channels' private step record ``char2 trajectory_vec[INTERCHANNEL_MAX_N_STEPS]``
   gets a large fixed capacity: the reference writes one entry per step and
   its first loop may take more steps than INTERCHANNEL_MAX_N_STEPS
   (opencl/connect.cl:48-76), which would overrun the array; only entries
   below INTERCHANNEL_MAX_N_STEPS-1 are ever read back (:80-97).

Each library exports ``slmref_run(void** args, uint n_global, uint offset,
int n_threads)``: it runs work-items ``offset .. offset+n_global-1`` of the
kernel, sequentially in ascending global id when ``n_threads == 1`` (the
pinned schedule) or with OpenMP otherwise, and ``slmref_P``.

The reference checkout is ``$SLM_REFERENCE`` when set, else ``reference/``
beside this repository's folder (``REFERENCE`` below).

Usage: python oracle/build_ref.py [--reference DIR] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# the reference checkout: $SLM_REFERENCE, else a "reference" folder beside the repository
REFERENCE = os.environ.get("SLM_REFERENCE") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
sys.path.insert(0, os.path.dirname(HERE))
from slm_b200.params import FIELDS  # noqa: E402

_TRACE = ["essentials.cl", "updatetraj.cl", "computestep.cl", "rungekutta.cl"]
# kernel function -> (KERNEL_ define, file list, where the reference builds it)
KERNELS = {
    "integrate_trajectory": ("INTEGRATE_TRAJECTORY",
        ["rng.cl", "essentials.cl", "writearray.cl", "updatetraj.cl", "computestep.cl",
         "rungekutta.cl", "trajectory.cl", "integratetraj.cl"], "trajectories.py:112-114"),
    "integrate_fields": ("INTEGRATE_FIELDS",
        ["rng.cl", "essentials.cl", "writearray.cl", "updatetraj.cl", "computestep.cl",
         "rungekutta.cl", "jittertrajectory.cl", "integratefields.cl"], "fields.py:103-106"),
    "connect_channels": ("CONNECT_CHANNELS", _TRACE + ["connect.cl"], "connect.py:48-50"),
    "map_channel_heads": ("MAP_CHANNEL_HEADS", _TRACE + ["channelheads.cl"], "channelheads.py:50-52"),
    "prune_channel_heads": ("PRUNE_CHANNEL_HEADS", _TRACE + ["channelheads.cl"], "channelheads.py:97-99"),
    "count_downchannels": ("COUNT_DOWNCHANNELS", _TRACE + ["countlink.cl"], "countlink.py:50-52"),
    "flag_downchannels": ("FLAG_DOWNCHANNELS",
        ["essentials.cl", "updatetraj.cl", "rungekutta.cl", "countlink.cl"], "countlink.py:98-99"),
    "label_confluences": ("LABEL_CONFLUENCES", ["essentials.cl", "updatetraj.cl", "label.cl"], "label.py:48-49"),
    "segment_downchannels": ("SEGMENT_DOWNCHANNELS",
        ["essentials.cl", "updatetraj.cl", "rungekutta.cl", "segment.cl"], "segment.py:52-53"),
    "segment_hillslopes": ("SEGMENT_HILLSLOPES", _TRACE + ["segment.cl"], "segment.py:113-115"),
    "subsegment_channel_edges": ("SUBSEGMENT_CHANNEL_EDGES", _TRACE + ["segment.cl"], "segment.py:166-168"),
    "subsegment_flanks": ("SUBSEGMENT_FLANKS", _TRACE + ["segment.cl"], "segment.py:166-168"),
    "fix_right_flanks": ("FIX_RIGHT_FLANKS", _TRACE + ["segment.cl"], "segment.py:166-168"),
    "fix_left_flanks": ("FIX_LEFT_FLANKS", _TRACE + ["segment.cl"], "segment.py:166-168"),
    "hillslopes": ("HILLSLOPES", _TRACE + ["hillslopes.cl"], "hillslopes.py:50-52"),
    "hillslope_lengths": ("HILLSLOPE_LENGTHS", _TRACE + ["lengths.cl"], "lengths.py:47-49"),
    "histogram_univariate": ("HISTOGRAM_UNIVARIATE", ["kde.cl"], "kde.py:138-142"),
    "histogram_bivariate": ("HISTOGRAM_BIVARIATE", ["kde.cl"], "kde.py:55-59"),
}
KDF_SHAPES = ["tophat", "triangle", "epanechnikov", "cosine", "gaussian"]
for _k in ("pdf_univariate", "pdf_bivariate_rows", "pdf_bivariate_cols"):
    for _s in KDF_SHAPES:
        KERNELS["{}__{}".format(_k, _s)] = (_k.upper(), ["kde.cl"], "kde.py:55-59,138-142")

CONNECT_CAP = 1 << 16


def lib_name(kernel):
    return os.path.join(OUT, "libref_{}.so".format(kernel))


def _match_paren(text, open_idx):
    depth = 0
    for i in range(open_idx, len(text)):
        c = text[i]
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced parenthesis")


def rewrite(src):
    """Apply the three syntactic rewrites described in the module docstring."""
    for vt in ("float2", "char2"):
        pat = "({})(".format(vt)
        while True:
            i = src.find(pat)
            if i < 0:
                break
            open_idx = i + len(pat) - 1
            close_idx = _match_paren(src, open_idx)
            src = (src[:i] + "(" + vt + "{" + src[open_idx + 1:close_idx] + "})" + src[close_idx + 1:])
    src = src.replace("(char)(", "slm_cvt_char(")
    src = re.sub(r"char2\s+trajectory_vec\[INTERCHANNEL_MAX_N_STEPS\]",
                 "char2 trajectory_vec[{}]".format(CONNECT_CAP), src)
    return src


def generate(kernel, reference):
    define, files, _cite = KERNELS[kernel]
    fn = kernel.split("__")[0]
    shape = kernel.split("__")[1] if "__" in kernel else None
    lines = ['#include "cl_shim.hpp"', "#include <utility>", "#include <omp.h>",
             'extern "C" {', "struct slmref_params {"]
    for name, kind in FIELDS:
        lines.append("    {} {};".format("uint" if kind == "u" else "float", name))
    lines += ["};", "slmref_params slmref_P;", "}"]
    for name, _kind in FIELDS:
        if name in ("do_measure_hsl_from_ridges", "kdf_kind"):
            continue
        lines.append("#define {} (slmref_P.{})".format(name.upper(), name))
    lines.append("#define KERNEL_{}".format(define))
    if shape:
        lines.append("#define KDF_IS_{}".format(shape.upper()))
    body = ""
    for f in files:
        with open(os.path.join(reference, "opencl", f)) as fp:
            body += fp.read()
    lines.append(rewrite(body))
    lines.append("""
template <class... A, std::size_t... I>
static void slmref_call_impl(void (*fn)(A...), void** args, std::index_sequence<I...>) {
    fn(((A)args[I])...);
}
template <class... A>
static void slmref_call(void (*fn)(A...), void** args) {
    slmref_call_impl(fn, args, std::index_sequence_for<A...>{});
}
extern "C" int slmref_run(void** args, uint n_global, uint offset, int n_threads) {
    slmref_gsize = n_global;
    slmref_goffset = offset;
    if (n_threads <= 1) {
        for (uint g = 0; g < n_global; ++g) {
            slmref_gid = offset + g;
            slmref_call(&%(fn)s, args);
        }
    } else {
        #pragma omp parallel for schedule(dynamic, 16) num_threads(n_threads)
        for (long g = 0; g < (long)n_global; ++g) {
            slmref_gid = offset + (uint)g;
            slmref_call(&%(fn)s, args);
        }
    }
    return 0;
}
""" % {"fn": fn})
    return "\n".join(lines) + "\n"


def build_one(kernel, reference, force=False):
    os.makedirs(OUT, exist_ok=True)
    src = generate(kernel, reference)
    shim = open(os.path.join(HERE, "cl_shim.hpp")).read()
    digest = hashlib.sha1((src + shim).encode()).hexdigest()[:16]
    cpp = os.path.join(OUT, "ref_{}.cpp".format(kernel))
    stamp = os.path.join(OUT, "ref_{}.sha1".format(kernel))
    so = lib_name(kernel)
    if not force and os.path.exists(so) and os.path.exists(stamp) \
            and open(stamp).read() == digest:
        return kernel, "cached"
    with open(cpp, "w") as fp:
        fp.write(src)
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp",
           "-ffp-contract=off", "-fno-fast-math", "-fno-strict-aliasing",
           "-w", "-I", HERE, cpp, "-o", so]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("g++ failed for {}:\n{}".format(kernel, r.stderr[-4000:]))
    with open(stamp, "w") as fp:
        fp.write(digest)
    os.remove(cpp)  # the generated source embeds the reference's; keep only the library
    return kernel, "built"


def build_all(reference=REFERENCE, jobs=8, force=False, only=None):
    if not os.path.isdir(os.path.join(reference, "opencl")):
        raise FileNotFoundError("reference checkout not found at {}".format(reference))
    names = [k for k in KERNELS if only is None or k.split("__")[0] in only or k in only]
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        return list(ex.map(lambda k: build_one(k, reference, force), names))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REFERENCE)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("kernels", nargs="*")
    a = ap.parse_args()
    for k, what in build_all(a.reference, a.jobs, a.force, a.kernels or None):
        print("{:32s} {}".format(k, what))
